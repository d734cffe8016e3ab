"""Times the reference's own CUDA solver (compiled from its sources by ``make -C oracle
ref`` into ``oracle/_ref/libxpbd_ref.so``) on a workload of this repository's scenes,
through the reference C ABI, on the current GPU.  Test infrastructure: a side-by-side
measurement, never part of the product path.

    python oracle/time_ref_gpu.py [--config large|plain] [--gaussians N] [--substeps K]

Prints one JSON line: ms per substep (blocking ``xpbd_step`` per substep with pins and
collider poses re-sent, as a caller does) and Gaussian-substeps/s.
"""
import argparse
import importlib
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libxpbd_ref.so")


def time_chainmail(args):
    """runChainmailGPU's dense path on the ChainMail workload: per step 30 seeds and the
    reference's default sweeps (20 propagation + 5 + 1 relax)."""
    import numpy as np
    n = args.gaussians or 1_000_000
    sc = pkg.scenes.chainmail_scene(n, 0)
    ref = pkg.bridge.XPBD(REF_SO)
    ref.create(sc)
    ref.step()
    ref.reset()
    pos = sc["pos"].astype(np.float64)

    def seeds(k):
        side = -1.0 if k % 2 == 0 else 1.0
        d = np.linalg.norm(pos - np.array([0.9 * side, 0.0, 0.0]), axis=1)
        return np.argpartition(d, 30)[:30].astype(np.int32), np.tile(np.float32([-0.005 * side, 0.0, 0.0]), (30, 1))

    cm = pkg.scenes.CHAINMAIL_DEFAULTS
    for k in range(3):
        ref.chainmail_seed(*seeds(k))
        ref.chainmail_run(**cm)
    steps = max(1, args.substeps // 4)
    t0 = time.perf_counter()
    for k in range(steps):
        ref.chainmail_seed(*seeds(k))
        ref.chainmail_run(**cm)
    dt = time.perf_counter() - t0
    sweeps = cm["prop_iters"] + cm["relax_iters"] + 1
    print(json.dumps({"impl": "reference CUDA (compiled from its sources)", "config": "chainmail", "n": n,
                      "steps": steps, "ms_per_step": dt / steps * 1e3,
                      "gauss_sweeps_per_s": n * sweeps * steps / dt}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="large", choices=["large", "plain", "chainmail"])
    ap.add_argument("--gaussians", type=int, default=None)
    ap.add_argument("--substeps", type=int, default=20)
    args = ap.parse_args()
    if args.config == "chainmail":
        return time_chainmail(args)
    if args.config == "plain":
        n = args.gaussians or 20000
        scen = pkg.scenes.plain_scene_scenario(n, 0)
    else:
        n = args.gaussians or 1_000_000
        scen = pkg.scenes.large_scene_scenario(n, 0)
    ref = pkg.bridge.XPBD(REF_SO)
    scen.setup(ref)
    scen.advance(ref, 11)                       # upload, topology build, warm-up
    t0 = time.perf_counter()
    scen.advance(ref, args.substeps)
    dt = time.perf_counter() - t0
    print(json.dumps({"impl": "reference CUDA (compiled from its sources)", "config": args.config, "n": n,
                      "substeps": args.substeps, "ms_per_substep": dt / args.substeps * 1e3,
                      "gauss_substeps_per_s": n * args.substeps / dt,
                      "self_collision_stats": [int(v) for v in ref.self_collision_stats()]}), flush=True)


if __name__ == "__main__":
    main()
