"""Shared test utilities: library paths, stage accessors, comparison metrics."""
import ctypes
import importlib
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")
scenes = pkg.scenes
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libxpbd_ref.so")
B200_SO = pkg.library_path()

# tolerances (fraction of the scene's bounding-box diagonal)
TOL_1STEP = 1e-5
TOL_100STEP = 1e-4


def ensure_oracle():
    if not os.path.isfile(ORACLE_SO):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    return ORACLE_SO


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


class Staged(pkg.bridge.XPBD):
    """XPBD bridge plus the stage accessors of the oracle (oracle_*), the product
    library (xpbd_b200_debug_*) or the reference shim (refshim_*)."""

    def __init__(self, path, prefix):
        self.CHAINMAIL_PREFIX = {"oracle": "oracle_", "b200": "xpbd_b200_", "ref": "refshim_"}[prefix]
        super().__init__(path)
        L = self.lib
        self.prefix = prefix
        names = {"oracle": ("oracle_int", "oracle_float", "oracle_selfcol_build"),
                 "b200": ("xpbd_b200_debug_int", "xpbd_b200_debug_float", "xpbd_b200_selfcol_build"),
                 "ref": ("refshim_int", "refshim_float", "refshim_selfcol_build")}[prefix]
        self._int, self._float, self._scb = (getattr(L, n) for n in names)
        for f in (self._int, self._float):
            f.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
            f.restype = ctypes.c_int
        self._scb.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._scb.restype = ctypes.c_int
        if prefix == "oracle":
            L.oracle_set_gs.argtypes = [ctypes.c_int, ctypes.c_int]
            L.oracle_set_volume_warp_mode.argtypes = [ctypes.c_int]
            L.oracle_set_threads.argtypes = [ctypes.c_int]
        elif prefix == "b200":
            L.xpbd_b200_set_gs.argtypes = [ctypes.c_int, ctypes.c_int]
            L.xpbd_b200_set_volume_warp_mode.argtypes = [ctypes.c_int]
            L.xpbd_b200_set_graph.argtypes = [ctypes.c_int]
        else:
            L.refshim_set_gs.argtypes = [ctypes.c_int, ctypes.c_int]

    def ints(self, name):
        n = self._int(name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(max(n, 1), np.int32)
        assert self._int(name.encode(), out.ctypes.data, out.size) == n
        return out[:n].copy()

    def floats(self, name):
        n = self._float(name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(max(n, 1), np.float32)
        assert self._float(name.encode(), out.ctypes.data, out.size) == n
        return out[:n].copy()

    def selfcol_build(self, x, p):
        x = np.ascontiguousarray(x, np.float32)
        p = np.ascontiguousarray(p, np.float32)
        return self._scb(x.ctypes.data, p.ctypes.data)

    def set_gs(self, dist, vol):
        fn = {"oracle": "oracle_set_gs", "b200": "xpbd_b200_set_gs", "ref": "refshim_set_gs"}[self.prefix]
        getattr(self.lib, fn)(int(dist), int(vol))

    def chainmail_times(self):
        if self.prefix != "ref":
            return super().chainmail_times()
        out = np.zeros(max(self.n, 1), np.float32)   # the reference keeps them in a file static
        assert self._float(b"cm_time", out.ctypes.data, out.size) == self.n
        return out[:self.n]

    def set_positions(self, pos):
        """Current positions (caller order), velocities kept: oracle_set_positions or
        xpbd_b200_set_positions."""
        fn = {"oracle": "oracle_set_positions", "b200": "xpbd_b200_set_positions"}[self.prefix]
        f = getattr(self.raw, fn)
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        f.restype = ctypes.c_int
        p = np.ascontiguousarray(pos, np.float32)
        self._check(getattr(self.lib, fn)(p.ctypes.data, len(p)), fn)


def oracle():
    return Staged(ensure_oracle(), "oracle")


def b200():
    return Staged(B200_SO, "b200")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def golden_scene(g):
    return {k[3:]: g[k] for k in g.files if k.startswith("in_")}


def scenario_for(case):
    """The scenario each golden case was generated with (tests/golden/make_golden.py)."""
    if case.startswith("plain_n4000"):
        kw = {}
        if case.endswith("_k1"):
            kw["ring_k"] = 1
        if case.endswith("_fpolar"):
            kw["shape_robust"] = False
        return scenes.plain_scene_scenario(4000, 3, pins=40, **kw)
    if case == "plain_n20000":
        return scenes.plain_scene_scenario(20000, 0)
    if case == "selfcol_blobs":
        return scenes.Scenario(*two_blob_scene(), self_collision=True, within_body=True)
    if case == "object_blobs":
        return scenes.Scenario(*two_blob_scene(), self_collision=True, within_body=False, object_shape=0.9)
    if case == "object_plain_n4000":
        return scenes.plain_scene_scenario(4000, 3, pins=40, object_shape=0.9)
    raise KeyError(case)


def two_blob_scene(n_each=1500):
    a = scenes.make_scene(n_each, 11, radii=(0.3, 0.3, 0.3), centre=(-0.35, 0.0, 0.0))
    b = scenes.make_scene(n_each, 12, radii=(0.3, 0.3, 0.3), centre=(0.35, 0.0, 0.0))
    sc = scenes.merge_scenes([a, b])
    grippers = [scenes.Gripper(sc["pos"], (-0.55, 0.0, 0.0), 60, (0.03, 0.0, 0.0)),
                scenes.Gripper(sc["pos"], (0.55, 0.0, 0.0), 60, (-0.03, 0.0, 0.0))]
    return sc, grippers


def max_err_over_diag(a, b, diag):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() / diag)


def covariances(scales, quats):
    """Sigma = R diag(s^2) R^T per Gaussian from (w, x, y, z) quaternions; invariant to the
    eigenvector sign and order choices of the shape writeback."""
    s = np.asarray(scales, np.float64)
    w, x, y, z = np.asarray(quats, np.float64).T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                  np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                  np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    return np.einsum("nij,nj,nkj->nik", R, s * s, R)


def covariance_rel_err(sa, qa, sb, qb):
    A, B = covariances(sa, qa), covariances(sb, qb)
    return np.linalg.norm((A - B).reshape(-1, 9), axis=1) / np.linalg.norm(B.reshape(-1, 9), axis=1)


def quat_angle(qa, qb):
    """Rotation angle between unit quaternions (sign-free), from the chord |qa - s qb| so that
    float32 rounding of the norms does not show as an angle (acos near 1 would)."""
    a = np.asarray(qa, np.float64)
    b = np.asarray(qb, np.float64)
    a = a / np.linalg.norm(a, axis=1, keepdims=True)
    b = b / np.linalg.norm(b, axis=1, keepdims=True)
    s = np.where((a * b).sum(1) < 0.0, -1.0, 1.0)[:, None]
    return 4.0 * np.arcsin(np.minimum(1.0, np.linalg.norm(a - s * b, axis=1) / 2.0))


# relative eigenvalue gap of Sigma below which a Gaussian's principal axes are
# ill-conditioned: an FP32 change of 1e-7 in Sigma turns them by more than 5e-6 rad, and
# two equal scales leave the axes in their plane undetermined
SHAPE_GAP = 2e-2


def shape_parity(sa, qa, sb, qb, diag):
    """Deformed-shape agreement of (scales, quats) a with reference b: max scale error over
    the bbox diagonal, max quaternion angle over the well-conditioned Gaussians (relative
    eigenvalue gap of Sigma >= SHAPE_GAP), the fraction exempt, and the max covariance
    relative error over the exempt ones."""
    sa, sb = np.asarray(sa, np.float64), np.asarray(sb, np.float64)
    lam = np.sort(sb * sb, axis=1)
    gap = np.minimum(lam[:, 1] - lam[:, 0], lam[:, 2] - lam[:, 1]) / lam[:, 2]
    good = gap >= SHAPE_GAP
    ang = quat_angle(qa, qb)
    cov = covariance_rel_err(sa, qa, sb, qb)
    return {"scale": float(np.abs(sa - sb).max() / diag),
            "angle": float(ang[good].max()) if good.any() else 0.0,
            "exempt": float(1.0 - good.mean()),
            "cov_exempt": float(cov[~good].max()) if (~good).any() else 0.0,
            "cov": float(cov.max())}


def press_run(solver, g):
    """tests/golden/make_golden.py's press script on the golden file's scene: the
    recorded press states and positions by tag."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    s = scenes.Scenario(golden_scene(g), [], substeps=1, iters=8)
    s.setup(solver)
    got = {}

    def record(tag, sv):
        got[f"state_{tag}"] = np.asarray(sv.press_state(), np.float32)
        if f"pos_{tag}" in g.files:
            got[f"pos_{tag}"] = sv.positions()
    mg.press_script(solver, record)
    return got


def runtime_scenario(g):
    """The runtime scenario a golden file holds, with its recorded grasp positions."""
    return scenes.RuntimeScenario(golden_scene(g), contact_bits=int(g["contact_bits"]), grasp_pos=g["grasp_pos"])


def cells_equal(start_a, end_a, start_b, end_b):
    """Cell ranges compared where a cell is occupied (the reference leaves stale ends in
    empty cells, forward.cu:11838)."""
    start_a, start_b = np.asarray(start_a), np.asarray(start_b)
    if not np.array_equal(start_a, start_b):
        return False
    occ = start_a >= 0
    return bool(np.array_equal(np.asarray(end_a)[occ], np.asarray(end_b)[occ]))


def contacts_equal(count_a, list_a, count_b, list_b):
    ca, cb = np.asarray(count_a), np.asarray(count_b)
    if not np.array_equal(ca, cb):
        return False
    la, lb = np.asarray(list_a).reshape(-1, 32), np.asarray(list_b).reshape(-1, 32)
    for i in np.nonzero(ca)[0]:
        if not np.array_equal(la[i, :ca[i]], lb[i, :ca[i]]):
            return False
    return True


# ---------------------------------------------------------------- splatting checkers
def cpu_render(fn, pos, scales, quats, opacity, colors, sh_degree, cam, scale_mod=1.0, antialias=False, box=None,
               bg=(0.0, 0.0, 0.0), pick=False, floor=None):
    """One frame through a stateless rasteriser with the oracle_render / refshim_render
    signature.  floor: None or (normal[3], height, origin[3], checker, fade)."""
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)   # noqa: E731
    P = ctypes.c_void_p
    fn.argtypes = ([ctypes.c_int] + [P] * 5 + [ctypes.c_int] + [P] * 3 + [ctypes.c_int, ctypes.c_int]
                   + [ctypes.c_float] * 3 + [ctypes.c_int] + [P] * 3 + [ctypes.c_int] + [P] * 6)
    fn.restype = ctypes.c_longlong
    n, W, H = len(pos), cam.width, cam.height
    arrs = [f32(pos), f32(scales), f32(quats), f32(opacity), f32(colors)]
    lo, hi = (f32(box[0]), f32(box[1])) if box is not None else (None, None)
    bgv = f32(bg)
    fl = None
    if floor is not None:
        fl = f32(list(floor[0]) + [floor[1]] + list(floor[2]) + [floor[3], floor[4]])
    out = np.zeros((3, H, W), np.float32)
    ft = np.zeros((H, W), np.float32)
    nc = np.zeros((H, W), np.int32)
    pk = np.full((H, W), -1, np.int32)
    radii = np.zeros(n, np.int32)
    ptr = lambda a: None if a is None else a.ctypes.data   # noqa: E731
    m = fn(n, *[a.ctypes.data for a in arrs], int(sh_degree), cam.view.ctypes.data, cam.proj.ctypes.data,
           cam.campos.ctypes.data, W, H, cam.tan_fovx, cam.tan_fovy, float(scale_mod), int(antialias), ptr(lo),
           ptr(hi), bgv.ctypes.data, int(pick), ptr(fl), out.ctypes.data, ft.ctypes.data, nc.ctypes.data,
           pk.ctypes.data, radii.ctypes.data)
    if m < 0:
        raise RuntimeError("render failed")
    return {"image": out, "final_T": ft, "n_contrib": nc, "pick": pk, "radii": radii, "pairs": int(m)}


def oracle_render(*args, **kw):
    lib = ctypes.CDLL(ensure_oracle())
    return cpu_render(lib.oracle_render, *args, **kw)


def image_diff(a, b):
    """(max |a-b|, mean |a-b|, fraction of values with |a-b| > 1e-3)."""
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    return float(d.max()), float(d.mean()), float((d > 1e-3).mean())
