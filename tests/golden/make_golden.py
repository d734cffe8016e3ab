"""Generate the golden fixtures in this folder from the reference solver itself.

Runs the reference's CUDA solver, compiled from its own sources by
``make -C oracle ref`` into ``oracle/_ref/libxpbd_ref.so`` (with the test-only accessor
shim ``oracle/ref_shim.cu``), through its own C ABI on seeded synthetic scenes, and
stores inputs and outputs as compressed ``.npz`` files.  It needs a GPU; the fixtures
it writes are committed so that the CPU oracle is pinned without one.

    python tests/golden/make_golden.py --out tests/golden

The reference prints its own diagnostics to stdout; they are not part of the output.
"""
import argparse
import ctypes
import importlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")
scenes = pkg.scenes
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libxpbd_ref.so")


class Ref(pkg.bridge.XPBD):
    """Reference library plus its accessor shim (oracle/ref_shim.cu)."""

    CHAINMAIL_PREFIX = "refshim_"

    def __init__(self):
        super().__init__(REF_SO)
        L = self.lib
        L.refshim_int.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
        L.refshim_int.restype = ctypes.c_int
        L.refshim_float.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
        L.refshim_float.restype = ctypes.c_int
        L.refshim_sizes.argtypes = [ctypes.c_void_p]
        L.refshim_set_gs.argtypes = [ctypes.c_int, ctypes.c_int]
        L.refshim_selfcol_build.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.refshim_selfcol_build.restype = ctypes.c_int

    def ints(self, name):
        n = self.lib.refshim_int(name.encode(), None, 0)
        if n < 0:
            raise RuntimeError(f"refshim_int({name}) unavailable")
        out = np.zeros(max(n, 1), np.int32)
        assert self.lib.refshim_int(name.encode(), out.ctypes.data, out.size) == n
        return out[:n].copy()

    def floats(self, name):
        n = self.lib.refshim_float(name.encode(), None, 0)
        if n < 0:
            raise RuntimeError(f"refshim_float({name}) unavailable")
        out = np.zeros(max(n, 1), np.float32)
        assert self.lib.refshim_float(name.encode(), out.ctypes.data, out.size) == n
        return out[:n].copy()

    def sizes(self):
        out = np.zeros(10, np.int64)
        self.lib.refshim_sizes(out.ctypes.data)
        return out

    def set_gs(self, dist, vol):
        self.lib.refshim_set_gs(int(dist), int(vol))

    def chainmail_times(self):
        return self.floats("cm_time")   # the reference keeps them in a file static

    def selfcol_build(self, x, p):
        x = np.ascontiguousarray(x, np.float32)
        p = np.ascontiguousarray(p, np.float32)
        return self.lib.refshim_selfcol_build(x.ctypes.data, p.ctypes.data)


def scene_arrays(sc):
    return {f"in_{k}": v for k, v in sc.items()}


def graph_case(ref, n, seed, ring_k, cap, leader):
    sc = scenes.make_scene(n, seed)
    s = scenes.Scenario(sc, [], ring_k=ring_k, max_members=cap, leader_min_hop=leader)
    s.setup(ref)
    ref.step()
    out = scene_arrays(sc)
    out.update(ring_k=ring_k, cap=cap, leader=leader, seed=seed)
    for name in ("nbr_offset", "nbr_count", "nbr_idx", "vol_offset", "vol_count", "vol_idx", "rev_offset",
                 "rev_count", "rev_idx", "mat_type", "gs_edge", "gs_color_offset", "vol_gs_order",
                 "vol_gs_color_offset", "obj_id"):
        try:
            out[name] = ref.ints(name)
        except RuntimeError:
            pass
    for name in ("det_rest", "sigma_rest", "v_rest", "rest_len", "gs_rest", "gs_stiff"):
        out[name] = ref.floats(name)
    out["pos_step1"] = ref.positions()
    return out


def scenario_case(ref, scen, checkpoints, gs=(0, 0), deform_eps=1e-3, vol_stats=True):
    scen.setup(ref)
    ref.set_gs(*gs)
    if vol_stats:
        ref.volume_stats(True)
    out = scene_arrays(scen.scene)
    out["pins_idx"] = np.concatenate([g.idx for g in scen.grippers]) if scen.grippers else np.zeros(0, np.int32)
    out["checkpoints"] = np.asarray(checkpoints, np.int64)
    t0 = time.time()
    done = 0
    for c in checkpoints:
        scen.advance(ref, c - done)
        done = c
        out[f"pos_{c}"] = ref.positions()
        out[f"vel_{c}"] = ref.floats("vel").reshape(-1, 3)
        if vol_stats:
            out[f"jvw_{c}"] = np.asarray(ref.volume_stats(True), np.float32)
        hits, push, cen = ref.collider_stats(len(scen.grippers))
        out[f"col_hits_{c}"] = hits
        out[f"col_push_{c}"] = push
        out[f"sc_stats_{c}"] = np.asarray(ref.self_collision_stats(), np.int32)
    sc_, q_, k_ = ref.shapes(deform_eps)
    out["shape_scales"] = sc_
    out["shape_quats"] = q_
    out["shape_deformed"] = np.int64(k_)
    out["deform_eps"] = np.float32(deform_eps)
    out["elapsed_s"] = np.float64(time.time() - t0)
    return out


def two_blob_scene(n_each=1500):
    a = scenes.make_scene(n_each, 11, radii=(0.3, 0.3, 0.3), centre=(-0.35, 0.0, 0.0))
    b = scenes.make_scene(n_each, 12, radii=(0.3, 0.3, 0.3), centre=(0.35, 0.0, 0.0))
    sc = scenes.merge_scenes([a, b])
    grippers = [scenes.Gripper(sc["pos"], (-0.55, 0.0, 0.0), 60, (0.03, 0.0, 0.0)),
                scenes.Gripper(sc["pos"], (0.55, 0.0, 0.0), 60, (-0.03, 0.0, 0.0))]
    return sc, grippers


def selfcol_case(ref, substeps_total=100):
    sc, grippers = two_blob_scene()
    scen = scenes.Scenario(sc, grippers, self_collision=True, within_body=True)
    out = scenario_case(ref, scen, [1, 50, substeps_total])
    # Stage-level fixture: the build on the final state, with predicted positions given.
    x = ref.positions()
    v = ref.floats("vel").reshape(-1, 3)
    p = (x + v * np.float32(scen.dt)).astype(np.float32)
    total = ref.selfcol_build(x, p)
    out["stage_x"] = x
    out["stage_p"] = p
    out["stage_total"] = np.int64(total)
    for name in ("sc_keys", "sc_keys_sorted", "sc_idx_sorted", "sc_cell_start", "sc_cell_end", "sc_contact",
                 "sc_count", "obj_id"):
        out[name] = ref.ints(name)
    out["self_col_params"] = ref.floats("self_col")
    out["table"] = np.int64(ref.sizes()[8])
    return out


def misc_case(ref):
    """Ground + gravity drop, launch with tilt, reset (forward.cu:4411-4446, 4551-4610, 7394-7599)."""
    sc = scenes.make_scene(2000, 5)
    scen = scenes.Scenario(sc, [])
    scen.setup(ref)
    out = scene_arrays(sc)
    ref.step()
    ref.set_ground(True, (0.0, 0.0, 1.0), -0.45, 0.5, 0.3, 0.0, 0.0, 9.8)
    ref.launch((0.0, 0.0, -1.0), (0.0, 0.0, 2.0), (0.3, 0.0, 0.0))
    out["pos_launch"] = ref.positions()
    for c in (1, 30, 90):
        while scen.k < c:
            ref.step()
            scen.k += 1
        out[f"pos_ground_{c}"] = ref.positions()
    ref.reset()
    out["pos_reset"] = ref.positions()
    ref.step()
    out["pos_after_reset_step"] = ref.positions()
    return out


def object_blobs_case(ref):
    """Object mode (forward.cu:12141-12166) on two objects pushed together by pinned
    grippers: weighted rigid fit, cross-object self-collision limited to the boxes of the
    other object, contact push."""
    sc, grippers = two_blob_scene()
    scen = scenes.Scenario(sc, grippers, self_collision=True, within_body=False, object_shape=0.9)
    return scenario_case(ref, scen, [1, 10, 30])


def chainmail_case(ref):
    """ChainMail waves through the reference's runChainmailGPU (forward.cu:12808-13006)."""
    sc = scenes.chainmail_scene(4000, 21)
    out = scene_arrays(sc)

    def record(tag):
        out[f"pos_{tag}"] = ref.positions()
        out[f"time_{tag}"] = ref.chainmail_times()

    scenes.chainmail_script(ref, sc, record)
    return out


RUNTIME_CHECKPOINTS = (1, 10, 30, 100)


def runtime_case(ref, contact_bits):
    """The Isaac runtime's configuration and call order (runtime_loop.py:39-71, 246-257,
    393-401, 519-548) through scenes.RuntimeScenario: 16 iterations at dt 1/60, leader
    spacing 2 with a 2048-member cap, object shape keeping, ellipsoid contacts, the ground
    with gravity and restitution, finger pads that close, hold and lift."""
    sc = scenes.make_scene(4000, 3)
    scen = scenes.RuntimeScenario(sc, contact_bits=contact_bits)
    out = scene_arrays(sc)
    out["contact_bits"] = np.int64(contact_bits)
    out["checkpoints"] = np.asarray(RUNTIME_CHECKPOINTS, np.int64)
    hits = []

    def record(solver, frame, shapes):
        hits.append(solver.collider_stats(2)[0])
        if frame in RUNTIME_CHECKPOINTS:
            out[f"pos_{frame}"] = solver.positions()
            out[f"vel_{frame}"] = ref.floats("vel").reshape(-1, 3)
            out[f"shape_scales_{frame}"], out[f"shape_quats_{frame}"] = shapes[0], shapes[1]
            out[f"shape_deformed_{frame}"] = np.int64(shapes[2])
    t0 = time.time()
    assert scen.setup(ref)
    scen.advance(ref, RUNTIME_CHECKPOINTS[-1], record)
    out["col_hits"] = np.asarray(hits, np.int32)
    out["grasp_pos"] = scen.grasp_pos
    out["vol_count"] = ref.ints("vol_count")
    out["elapsed_s"] = np.float64(time.time() - t0)
    return out


PRESS_CHECKPOINTS = (1, 10, 40)


def press_script(solver, record):
    """Press harness through the C ABI (xpbd_capi.cu:281-303; forward.cu:4311-4409,
    9411-9424, 12095-12111): a plate closing down the z axis at 1.2/s without settling
    pauses, stopped; then one closing up from below at 3/s with the 25/50/75/100 %
    pauses (the first one ends within the run); then reset.  record(tag, solver) after
    the marked steps."""
    solver.step()
    solver.press_autolog(False)
    solver.press_start(2, 1.2, 0.4, 0)
    record("start", solver)
    for k in range(1, PRESS_CHECKPOINTS[-1] + 1):
        solver.step()
        if k in PRESS_CHECKPOINTS:
            record(f"a{k}", solver)
    solver.press_stop()
    solver.step()
    record("stopped", solver)
    solver.press_autolog(True)
    solver.press_start(2, 3.0, 0.5, 1)
    for k in range(1, 101):          # the 25 % pause (90 steps) ends at step 93
        solver.step()
        record(f"b{k}", solver)
    solver.reset()
    record("reset", solver)
    solver.press_autolog(True)


def press_case(ref):
    sc = scenes.make_scene(3000, 7)
    scen = scenes.Scenario(sc, [], substeps=1, iters=8)
    scen.setup(ref)
    out = scene_arrays(sc)

    def record(tag, solver):
        out[f"state_{tag}"] = np.asarray(solver.press_state(), np.float32)
        if tag in ("a1", "a10", "a40", "stopped", "b100"):
            out[f"pos_{tag}"] = solver.positions()
    press_script(ref, record)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    names = ["graph_n3000_r1", "graph_n3000_r2", "graph_n3000_k1", "plain_n4000", "plain_n4000_k1",
             "plain_n4000_fpolar", "plain_n4000_gs", "plain_n20000", "selfcol_blobs", "misc_n2000", "chainmail_n4000", "object_blobs",
             "object_plain_n4000", "runtime_n4000", "runtime_n4000_ground", "press_n3000"]
    if not args.only:
        # One process per case: the reference keeps its solver state in file-static globals.
        import subprocess
        rc = 0
        for name in names:
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--out", args.out, "--only", name],
                               stdout=subprocess.DEVNULL)
            print(f"[golden] {name}: exit {r.returncode}", file=sys.stderr, flush=True)
            rc = rc or r.returncode
        sys.exit(rc)
    ref = Ref()
    cases = {
        "graph_n3000_r1": lambda: graph_case(ref, 3000, 1, 3, 64, 1),
        "graph_n3000_r2": lambda: graph_case(ref, 3000, 1, 3, 64, 2),
        "graph_n3000_k1": lambda: graph_case(ref, 3000, 1, 1, 64, 1),
        "plain_n4000": lambda: scenario_case(ref, scenes.plain_scene_scenario(4000, 3, pins=40), [1, 10, 100]),
        "plain_n4000_k1": lambda: scenario_case(
            ref, scenes.plain_scene_scenario(4000, 3, pins=40, ring_k=1), [1, 10, 100]),
        "plain_n4000_fpolar": lambda: scenario_case(
            ref, scenes.plain_scene_scenario(4000, 3, pins=40, shape_robust=False), [1, 10, 100]),
        "plain_n4000_gs": lambda: scenario_case(
            ref, scenes.plain_scene_scenario(4000, 3, pins=40), [1, 10, 100], gs=(1, 1)),
        "plain_n20000": lambda: scenario_case(ref, scenes.plain_scene_scenario(20000, 0), [1, 100, 1000]),
        "selfcol_blobs": lambda: selfcol_case(ref),
        "misc_n2000": lambda: misc_case(ref),
        "chainmail_n4000": lambda: chainmail_case(ref),
        "object_blobs": lambda: object_blobs_case(ref),
        "object_plain_n4000": lambda: scenario_case(
            ref, scenes.plain_scene_scenario(4000, 3, pins=40, object_shape=0.9), [1, 10, 100]),
        "runtime_n4000": lambda: runtime_case(ref, 1),
        "runtime_n4000_ground": lambda: runtime_case(ref, 3),
        "press_n3000": lambda: press_case(ref),
    }
    for name, fn in cases.items():
        if args.only and name not in args.only.split(","):
            continue
        t0 = time.time()
        data = fn()
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **data)
        print(f"[golden] {name}: {time.time() - t0:.1f}s", file=sys.stderr, flush=True)
        ref.destroy()


if __name__ == "__main__":
    main()
