"""Cameras for the library's splatting pass (``xpbd_b200_render``).

The rasteriser takes the 3DGS camera of the reference viewer: a world->view matrix
(view space x right, y down, z forward) and a full world->clip matrix, both passed
column-major, plus tan of the half fields of view.  The projection is the 3DGS one
(getProjectionMatrix of the Gaussian-splatting code base: z_sign +1, depth mapped to
[0, 1]); ``Camera.look_at`` builds all of it from an eye point, a target and an up
vector.
"""
import math
from dataclasses import dataclass

import numpy as np


def _normalize(v):
    v = np.asarray(v, np.float64)
    n = np.linalg.norm(v)
    if not n > 0:
        raise ValueError("zero-length vector")
    return v / n


def projection(znear, zfar, fovx, fovy):
    """The 3DGS perspective matrix (row-major, acting on column vectors)."""
    tx, ty = math.tan(fovx / 2), math.tan(fovy / 2)
    top, bottom, right, left = ty * znear, -ty * znear, tx * znear, -tx * znear
    P = np.zeros((4, 4), np.float64)
    P[0, 0] = 2 * znear / (right - left)
    P[1, 1] = 2 * znear / (top - bottom)
    P[0, 2] = (right + left) / (right - left)
    P[1, 2] = (top + bottom) / (top - bottom)
    P[3, 2] = 1.0
    P[2, 2] = zfar / (zfar - znear)
    P[2, 3] = -(zfar * znear) / (zfar - znear)
    return P


@dataclass
class Camera:
    width: int
    height: int
    view: np.ndarray      # (16,) float32, column-major world -> view
    proj: np.ndarray      # (16,) float32, column-major world -> clip (projection @ view)
    campos: np.ndarray    # (3,) float32
    tan_fovx: float
    tan_fovy: float

    @staticmethod
    def look_at(eye, target, up, width, height, fovy_deg=50.0, znear=0.01, zfar=100.0):
        eye = np.asarray(eye, np.float64)
        f = _normalize(np.asarray(target, np.float64) - eye)
        u = np.asarray(up, np.float64)
        d = _normalize(-(u - np.dot(u, f) * f))       # image down
        r = np.cross(d, f)                             # x = y cross z
        V = np.eye(4)
        V[0, :3], V[1, :3], V[2, :3] = r, d, f
        V[:3, 3] = -V[:3, :3] @ eye
        fovy = math.radians(fovy_deg)
        fovx = 2 * math.atan(math.tan(fovy / 2) * width / height)
        P = projection(znear, zfar, fovx, fovy) @ V
        return Camera(int(width), int(height), V.T.astype(np.float32).ravel().copy(),
                      P.T.astype(np.float32).ravel().copy(), eye.astype(np.float32),
                      math.tan(fovx / 2), math.tan(fovy / 2))

    @staticmethod
    def framing(points, width, height, direction=(0.3, -1.0, 0.5), up=(0.0, 0.0, 1.0), fovy_deg=50.0, margin=1.3):
        """A camera that looks at the centre of ``points`` from ``direction``, far
        enough back for the bounding sphere to fill the view."""
        p = np.asarray(points, np.float64)
        c = 0.5 * (p.min(0) + p.max(0))
        rad = 0.5 * float(np.linalg.norm(p.max(0) - p.min(0))) * margin
        dist = rad / math.sin(math.radians(fovy_deg) / 2)
        eye = c - _normalize(direction) * dist
        return Camera.look_at(eye, c, up, width, height, fovy_deg, znear=0.01, zfar=max(100.0, 4 * dist))


def synthetic_colors(n, sh_degree=-1, seed=0):
    """Seeded colours: RGB in [0.1, 0.9] (sh_degree -1) or SH coefficients (n,
    (d+1)^2, 3) whose DC term gives the same range and whose higher bands add a
    view-dependent tint of a few percent."""
    rng = np.random.default_rng(seed)
    rgb = rng.uniform(0.1, 0.9, (n, 3)).astype(np.float32)
    if sh_degree < 0:
        return rgb
    m = (sh_degree + 1) ** 2
    sh = np.zeros((n, m, 3), np.float32)
    sh[:, 0, :] = (rgb - 0.5) / 0.28209479177387814
    if m > 1:
        sh[:, 1:, :] = rng.normal(0.0, 0.05, (n, m - 1, 3))
    return sh
