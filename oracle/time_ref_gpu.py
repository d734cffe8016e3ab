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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="large", choices=["large", "plain"])
    ap.add_argument("--gaussians", type=int, default=None)
    ap.add_argument("--substeps", type=int, default=20)
    args = ap.parse_args()
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
