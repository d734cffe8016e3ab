"""The one-pass moment forms that the volume-cluster solve and shape matching use in
place of the reference's two-pass centred sums, checked in FP32 on the clusters and
1-rings of a seeded scene against the same sums in FP64 (CPU; the GPU parity tests
compare the kernels themselves with the oracle).

Volume cluster (leader p, members q_k, d_k = q_k - p, c' = c - p):
    Sigma = sum_{k in members + leader} (q_k - c)(q_k - c)^T / (m+1)
          = sum d d^T / (m+1) - c' c'^T
    sum_k w_k |g Sinv (q_k - c)|^2 = g^2 tr(Sinv^2 W),
    W = sum w d d^T - c' (sum w d)^T - (sum w d) c'^T + (sum w) c' c'^T
Shape matching (Gaussian i, neighbours j, dq = q - p_i, dr = r - r_i):
    A = sum (q - com)(r - com_rest)^T
      = sum dq dr^T - cq (sum dr)^T - (sum dq) cr^T + (m+1) cq cr^T
"""
import importlib

import numpy as np

pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")


def neighbourhoods(n=4000, k=64, seed=2):
    from scipy.spatial import cKDTree

    sc = pkg.scenes.make_scene(n, seed)
    pos = sc["pos"].astype(np.float64)
    _, nn = cKDTree(pos).query(pos, k=k + 1)
    rng = np.random.default_rng(seed)
    cur = pos + rng.normal(0.0, 0.002, pos.shape)       # a deformed state
    w = rng.uniform(0.0, 1.0, n)
    return pos, cur, w, nn


def test_volume_moment_form_matches_centred_sums():
    _, cur, w, nn = neighbourhoods()
    worst_cov, worst_den = 0.0, 0.0
    for i in range(0, len(cur), 37):
        pts = cur[nn[i]]                                  # leader first, then 64 members
        ws = w[nn[i]]
        # reference: centred two-pass in FP64
        c = pts.mean(0)
        cov = (pts - c).T @ (pts - c) / len(pts)
        sinv = np.linalg.inv(cov + 1e-9 * np.eye(3))
        den = sum(ws[k] * np.sum((sinv @ (pts[k] - c)) ** 2) for k in range(len(pts)))
        # moment form in FP32, relative to the leader
        p = pts[0].astype(np.float32)
        d = pts[1:].astype(np.float32) - p
        wm = ws[1:].astype(np.float32)
        inv_n = np.float32(1.0) / np.float32(len(pts))
        cp = d.sum(0, dtype=np.float32) * inv_n
        cov32 = (d.T @ d).astype(np.float32) * inv_n - np.outer(cp, cp)
        wd = (wm[:, None] * d).sum(0, dtype=np.float32)
        wdd = (d.T * wm) @ d
        wsum = wm.sum(dtype=np.float32) + np.float32(ws[0])
        W = wdd - np.outer(cp, wd) - np.outer(wd, cp) + wsum * np.outer(cp, cp)
        sinv32 = sinv.astype(np.float32)
        den32 = float(np.sum((sinv32 @ sinv32) * W))
        worst_cov = max(worst_cov, float(np.abs(cov32 - cov).max() / np.abs(cov).max()))
        worst_den = max(worst_den, abs(den32 - den) / den)
    assert worst_cov < 1e-5, worst_cov
    assert worst_den < 1e-5, worst_den


def test_shape_moment_form_matches_centred_sums():
    rest, cur, _, nn = neighbourhoods(k=9)
    worst = 0.0
    for i in range(0, len(cur), 13):
        q, r = cur[nn[i]], rest[nn[i]]                    # the Gaussian first, then its 1-ring
        A = (q - q.mean(0)).T @ (r - r.mean(0))
        q32, r32 = q.astype(np.float32), r.astype(np.float32)
        dq, dr = q32[1:] - q32[0], r32[1:] - r32[0]
        cq = q32.sum(0, dtype=np.float32) / np.float32(len(q)) - q32[0]
        cr = r32.sum(0, dtype=np.float32) / np.float32(len(r)) - r32[0]
        A32 = (dq.T @ dr - np.outer(cq, dr.sum(0)) - np.outer(dq.sum(0), cr)
               + np.float32(len(q)) * np.outer(cq, cr))
        worst = max(worst, float(np.abs(A32 - A).max() / np.abs(A).max()))
    assert worst < 1e-5, worst
