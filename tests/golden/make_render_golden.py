"""Golden frames of the reference's own rasteriser for the splatting parity tests.

Runs the reference viewer's preprocessCUDA / renderCUDA (compiled from its sources into
oracle/_ref/libxpbd_ref.so, entry point refshim_render) on seeded Gaussian sets and
cameras, and writes inputs and outputs to one .npz.  Needs a CUDA GPU and the reference
build; the file it writes is committed as tests/golden/render_ref.npz.

    python tests/golden/make_render_golden.py [out.npz]
"""
import ctypes
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
import helpers  # noqa: E402

pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")

# (name, n, seed, sh_degree, width, height, view direction, antialias, box, pick, floor)
CASES = [
    ("rgb", 1500, 31, -1, 128, 96, (0.3, -1.0, 0.5), False, False, True, False),
    ("sh3_aa", 1500, 32, 3, 100, 70, (-0.6, -1.0, -0.2), True, False, False, False),
    ("sh1_box_floor", 1500, 33, 1, 96, 96, (0.2, 1.0, -0.8), False, True, True, True),
]


def case_inputs(n, seed, sh_degree, width, height, direction):
    sc = pkg.scenes.make_scene(n, seed, radii=(0.5, 0.35, 0.3))
    colors = pkg.splat.synthetic_colors(n, sh_degree, seed + 100)
    cam = pkg.splat.Camera.framing(sc["pos"], width, height, direction=direction)
    return sc, colors, cam


def main(out_path):
    lib = ctypes.CDLL(helpers.REF_SO)
    data = {}
    for name, n, seed, deg, W, H, direction, aa, box, pick, floor in CASES:
        sc, colors, cam = case_inputs(n, seed, deg, W, H, direction)
        bx = ((-0.3, -0.5, -0.5), (0.3, 0.5, 0.5)) if box else None
        fl = ((0.0, 0.0, 1.0), -0.4, (0.0, 0.0, -0.4), 0.15, 3.0) if floor else None
        r = helpers.cpu_render(lib.refshim_render, sc["pos"], sc["scales"], sc["rots"], sc["opacity"], colors, deg,
                               cam, antialias=aa, box=bx, bg=(0.1, 0.2, 0.3), pick=pick, floor=fl)
        for k, v in r.items():
            data[f"{name}/{k}"] = np.asarray(v)
        print(f"{name}: pairs {r['pairs']}, visible {(r['radii'] > 0).sum()}, "
              f"coverage {(r['final_T'] < 0.5).mean():.2f}")
    np.savez_compressed(out_path, **data)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "render_ref.npz"))
