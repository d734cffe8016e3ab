"""Graph and splat file formats of the reference pipeline.

* ``APGGRPH1`` — the physics graph a viewer exports (exportPhysicsGraph,
  forward.cu:4612-4663): little endian ``"APGGRPH1" | int32 N | int32 M |
  float32 pos_rest[N*3] | int32 offset[N] | int32 count[N] | int32 idx[M] |
  float32 dist[M] | float32 stiff[M]`` (a directed CSR, both directions of every edge).
  ``read_graph`` / ``write_graph``; the library writes one with
  ``xpbd_b200_export_graph`` (in the order given to ``xpbd_create``).
* The graph ``.npz`` the runtime loads (tools/import_graph.py:124-126): the same CSR
  renumbered into the splat file's order by matching rest positions bit for bit, plus
  ``pos_rest`` and ``sibr_to_usd``.  ``reorder_graph`` does the renumbering,
  ``save_graph_npz`` / ``load_graph_npz`` the file.
* 3DGS binary PLY (``x y z``, ``scale_0..2`` in log space, ``rot_0..3``, ``opacity`` as a
  logit, any other float properties): ``read_ply`` / ``write_ply``.
* ``load_inputs`` turns a splat PLY and its graph ``.npz`` into the ``xpbd_create``
  arrays exactly as the reference bridge does (src/xpbd_bridge.py:18-42): activated
  scales, normalised quaternions, sigmoid opacity, undirected edges i < j.
"""
import os

import numpy as np

MAGIC = b"APGGRPH1"


# ---------------------------------------------------------------------------- APGGRPH1
def read_graph(path):
    """(N, M, {"pos", "offset", "count", "idx", "dist", "stiff"}) of an APGGRPH1 file."""
    raw = open(path, "rb").read()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not an APGGRPH1 file (magic {raw[:8]!r})")
    n, m = (int(v) for v in np.frombuffer(raw, dtype="<i4", count=2, offset=8))
    at = 16
    out = {}
    for name, dtype, count in (("pos", "<f4", 3 * n), ("offset", "<i4", n), ("count", "<i4", n),
                               ("idx", "<i4", m), ("dist", "<f4", m), ("stiff", "<f4", m)):
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=at)
        at += a.nbytes
        out[name] = a.reshape(n, 3).copy() if name == "pos" else a.copy()
    if at != len(raw):
        raise ValueError(f"{path}: {len(raw)} bytes, the header says {at}")
    return n, m, out


def write_graph(path, pos, offset, count, idx, dist, stiff):
    pos = np.ascontiguousarray(pos, dtype="<f4").reshape(-1, 3)
    n, m = pos.shape[0], int(len(idx))
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.asarray([n, m], dtype="<i4").tobytes())
        for a, dt in ((pos, "<f4"), (offset, "<i4"), (count, "<i4"), (idx, "<i4"), (dist, "<f4"), (stiff, "<f4")):
            f.write(np.ascontiguousarray(a, dtype=dt).tobytes())


def scene_csr(scene):
    """The directed CSR of a scene's undirected edges in loadGraph's order: every edge
    lands in both endpoints' rows, rows filled in edge order (forward.cu:2702-2779)."""
    n = scene["pos"].shape[0]
    e = np.asarray(scene["edges"], dtype=np.int64).reshape(-1, 2)
    ok = (e[:, 0] >= 0) & (e[:, 1] >= 0) & (e[:, 0] < n) & (e[:, 1] < n) & (e[:, 0] != e[:, 1])
    e = e[ok]
    rest = np.asarray(scene["rest"], np.float32)[ok]
    stiff = np.asarray(scene["stiff"], np.float32)[ok]
    ends = np.stack([e[:, 0], e[:, 1]], axis=1).ravel()      # a0, b0, a1, b1, ...
    other = np.stack([e[:, 1], e[:, 0]], axis=1).ravel()
    edge = np.repeat(np.arange(len(e)), 2)
    order = np.argsort(ends, kind="stable")
    count = np.bincount(ends, minlength=n)
    offset = np.zeros(n, np.int64)
    offset[1:] = np.cumsum(count)[:-1]
    return (offset.astype(np.int32), count.astype(np.int32), other[order].astype(np.int32),
            rest[edge[order]], stiff[edge[order]])


# ------------------------------------------------------------------ viewer -> splat order
def _keys(p):
    return np.ascontiguousarray(p, dtype=np.float32).view(np.dtype((np.void, 12))).ravel()


def reorder_graph(g, pos_target):
    """The CSR of ``g`` (read_graph) renumbered into the order of ``pos_target`` (N, 3)
    by matching rest positions bit for bit (tools/import_graph.py:73-118).  Returns the
    .npz fields: offset, count, idx, dist, stiff, pos_rest, sibr_to_usd."""
    pos_target = np.asarray(pos_target, np.float32)
    n = g["pos"].shape[0]
    if pos_target.shape[0] != n:
        raise ValueError(f"graph has {n} nodes, the splats {pos_target.shape[0]}")
    kt, kg = _keys(pos_target), _keys(g["pos"])
    uniq, first, cnt = np.unique(kt, return_index=True, return_counts=True)
    at = np.clip(np.searchsorted(uniq, kg), 0, len(uniq) - 1)
    if not (uniq[at] == kg).all():
        raise ValueError(f"{int((uniq[at] != kg).sum())} graph nodes have no bit-identical splat position")
    g2t = first[at].astype(np.int64)
    if len(np.unique(g2t)) != n:
        raise ValueError("the position match is not one to one (repeated positions)")
    t2g = np.empty(n, np.int64)
    t2g[g2t] = np.arange(n)
    off_g, cnt_g = g["offset"].astype(np.int64), g["count"].astype(np.int64)
    count = cnt_g[t2g]
    offset = np.zeros(n, np.int64)
    offset[1:] = np.cumsum(count)[:-1]
    gather = (np.concatenate([np.arange(off_g[s], off_g[s] + cnt_g[s]) for s in t2g])
              if count.sum() else np.zeros(0, np.int64))
    idx_g = g["idx"][gather].astype(np.int64)
    valid = (idx_g >= 0) & (idx_g < n)
    idx = np.where(valid, g2t[np.clip(idx_g, 0, n - 1)], -1).astype(np.int32)
    return {"offset": offset.astype(np.int32), "count": count.astype(np.int32), "idx": idx,
            "dist": g["dist"][gather].astype(np.float32), "stiff": g["stiff"][gather].astype(np.float32),
            "pos_rest": pos_target, "sibr_to_usd": g2t.astype(np.int32)}


def save_graph_npz(path, fields):
    np.savez_compressed(path, **fields)


def load_graph_npz(path):
    g = np.load(path)
    return {k: g[k] for k in g.files}


# ---------------------------------------------------------------------------- 3DGS PLY
_PLY_TYPES = {"float": "<f4", "float32": "<f4", "double": "<f8", "uchar": "u1", "uint8": "u1", "int": "<i4",
              "int32": "<i4", "uint": "<u4", "short": "<i2", "ushort": "<u2", "char": "i1"}


def read_ply(path):
    """(count, {property: array}) of the vertex element of a binary little-endian PLY."""
    with open(path, "rb") as f:
        header = []
        while True:
            line = f.readline()
            if not line:
                raise ValueError(f"{path}: no end_header")
            line = line.decode("ascii").strip()
            header.append(line)
            if line == "end_header":
                break
        body = f.read()
    if "format binary_little_endian 1.0" not in header:
        raise ValueError(f"{path}: only binary_little_endian PLY is read")
    count, props, in_vertex = 0, [], False
    for line in header:
        w = line.split()
        if w[:2] == ["element", "vertex"]:
            count, in_vertex = int(w[2]), True
        elif w and w[0] == "element":
            in_vertex = False
        elif in_vertex and w[:1] == ["property"]:
            if w[1] == "list":
                raise ValueError(f"{path}: list properties in the vertex element are not read")
            props.append((w[2], _PLY_TYPES[w[1]]))
    rec = np.frombuffer(body, dtype=np.dtype(props), count=count)
    return count, {name: np.asarray(rec[name]) for name, _ in props}


def write_ply(path, data):
    """Binary little-endian PLY with one float32 vertex property per dict entry."""
    names = list(data)
    n = len(data[names[0]])
    rec = np.empty(n, dtype=[(k, "<f4") for k in names])
    for k in names:
        rec[k] = data[k]
    head = ["ply", "format binary_little_endian 1.0", f"element vertex {n}"]
    head += [f"property float {k}" for k in names] + ["end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode("ascii"))
        f.write(rec.tobytes())


def splat_fields(scene):
    """The 3DGS PLY fields of a scene dict (log scales, logit opacity)."""
    s = np.log(np.asarray(scene["scales"], np.float64))
    a = np.clip(np.asarray(scene["opacity"], np.float64), 1e-7, 1 - 1e-7)
    out = {"x": scene["pos"][:, 0], "y": scene["pos"][:, 1], "z": scene["pos"][:, 2]}
    for i in range(3):
        out[f"scale_{i}"] = s[:, i]
    for i in range(4):
        out[f"rot_{i}"] = scene["rots"][:, i]
    out["opacity"] = np.log(a / (1 - a))
    return {k: np.asarray(v, np.float32) for k, v in out.items()}


# ---------------------------------------------------------------------- runtime inputs
def load_inputs(d, name):
    """``xpbd_create`` arrays from <d>/<name>_crop.ply and <d>/<name>_graph.npz (both in
    splat order), as the reference bridge builds them (src/xpbd_bridge.py:18-42)."""
    _, data = read_ply(os.path.join(d, f"{name}_crop.ply"))
    g = load_graph_npz(os.path.join(d, f"{name}_graph.npz"))
    pos = np.stack([data["x"], data["y"], data["z"]], axis=1).astype(np.float32)
    if not np.array_equal(pos, g["pos_rest"]):
        raise ValueError("graph pos_rest differs from the splat positions: renumber the graph again")
    scales = np.exp(np.stack([data["scale_0"], data["scale_1"], data["scale_2"]], axis=1)).astype(np.float32)
    rots = np.stack([data["rot_0"], data["rot_1"], data["rot_2"], data["rot_3"]], axis=1).astype(np.float32)
    rots /= np.linalg.norm(rots, axis=1, keepdims=True)
    opacity = (1.0 / (1.0 + np.exp(-data["opacity"].astype(np.float64)))).astype(np.float32)
    owner = np.repeat(np.arange(len(pos), dtype=np.int32), g["count"])
    keep = g["idx"] > owner
    return {
        "pos": np.ascontiguousarray(pos),
        "scales": np.ascontiguousarray(scales),
        "rots": np.ascontiguousarray(rots),
        "opacity": np.ascontiguousarray(opacity),
        "edges": np.ascontiguousarray(np.stack([owner[keep], g["idx"][keep]], axis=1).astype(np.int32)),
        "rest": np.ascontiguousarray(g["dist"][keep].astype(np.float32)),
        "stiff": np.ascontiguousarray(g["stiff"][keep].astype(np.float32)),
    }
