"""Throughput benchmark of the XPBD Gaussian-graph step (one JSON line on rank 0).

Workload (default): the large single scene — 1,000,000 Gaussians (ellipsoid, 8-NN
graph, 64-member volume clusters, shape matching, spatial-hash self-collision), two
capsule grippers pulling apart while twisting; one bench "step" is one 60 Hz frame =
10 solver substeps x 4 iterations.  Metric: Gaussian-substeps per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--config large|plain|batched|served|chainmail|dense|render]
                  [--gaussians N]

value     device-resident throughput: frames enqueued through the library's async API
          (one xpbd_b200_step_substeps call per frame, one CUDA-graph replay per
          substep), timed with CUDA events on the engine's stream (pins/colliders
          re-posed per substep from host, as a caller does);
e2e       the same frames through the reference-facing C ABI (xpbd_set_colliders /
          xpbd_set_attached / blocking xpbd_step per substep, xpbd_positions_host per frame);
roofline  the dominant kernel's algorithmic bytes / its mean CUDA-event duration, from
          the timed frames repeated with an event pair around every kernel, against the
          measured HBM copy bandwidth;
cpu_baseline  the CPU oracle (OpenMP, all host cores) on a bounded sample;
reference_gpu the reference's own CUDA solver compiled from its sources (oracle/_ref) on
          the same workload and GPU, ms per substep and the ratio;
batched, served  (default large config, one GPU) the batched 64-object and served
          halves of the headline metric at reduced step counts, each with its plain
          one-scene-at-a-time comparison (--config batched / served run them alone).

--impl reference times the reference's CPU path.  The reference has no CPU XPBD
solver, so this is the C restatement oracle/liboracle.so with all host threads; each
"step" is one substep of the same workload.  Multi-GPU (torchrun): every rank runs an
independent replica (the step has no exchange), barrier + max over ranks.
"""
import argparse
import ctypes
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
pkg = importlib.import_module("3dgs-isaac-sim-xpbd_b200")
scenes = pkg.scenes

METRIC = "XPBD substeps/s at 1M Gaussians (Gaussian-substeps/s)"
UNIT = "Gaussian-substeps/s"
SUBSTEPS = 10
ITERS = 4


def workload(config, gaussians=None):
    """(name, scenario factory) of a single-scene workload; `gaussians` shrinks or grows
    the scene (profiler captures use a small case of the same workload)."""
    if config == "dense":
        n = gaussians or 4_000_000
        return (f"dense contact: {n} Gaussians, 12-NN graph, 128-member clusters (k=3), shape matching, "
                "self-collision, two plates closing 0.005 per frame, 10 substeps x 20 iterations"), \
            lambda: scenes.dense_contact_scenario(n, 0)
    if config == "plain":
        n = gaussians or 20000
        return f"plain: {n} Gaussians, 2 pinned capsule grippers, 10 substeps x 4 iterations", \
            lambda: scenes.plain_scene_scenario(n, 0)
    n = gaussians or 1_000_000
    return (f"large: {n} Gaussians, 8-NN graph, 64-member clusters (k=3), shape matching, "
            "spatial-hash self-collision, 2 twisting grippers, 10 substeps x 4 iterations"), \
        lambda: scenes.large_scene_scenario(n, 0)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.first = threading.Event()
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            self.first.wait(3.0)      # sampling is running before the timed region starts
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())
            self.first.set()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def bind_ext(L):
    L.xpbd_b200_set_stream.argtypes = [ctypes.c_void_p]
    L.xpbd_b200_step_async.argtypes = [ctypes.c_int]
    L.xpbd_b200_set_profiling.argtypes = [ctypes.c_int]
    L.xpbd_b200_stage_times.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.xpbd_b200_stage_name.restype = ctypes.c_char_p
    L.xpbd_b200_stage_name.argtypes = [ctypes.c_int]
    L.xpbd_b200_launch_count.restype = ctypes.c_longlong
    L.xpbd_b200_sizes.argtypes = [ctypes.c_void_p]
    L.xpbd_b200_set_fused.argtypes = [ctypes.c_int]
    L.xpbd_b200_tuning.argtypes = [ctypes.c_void_p]


FORMS = ("kernel sequence", "fused cooperative launch", "sequence, volume kernels at 6 blocks/SM",
         "sequence, volume kernels at 8 blocks/SM")


def tuning(L):
    """The step form the autotuner chose and the mean trial-step times of every form."""
    t = np.zeros(7, np.float32)
    L.xpbd_b200_tuning(t.ctypes.data)
    ms = {FORMS[0]: float(t[2]), FORMS[1]: float(t[3]), FORMS[2]: float(t[5]), FORMS[3]: float(t[6])}
    return {"form": FORMS[int(t[0])], "decided": bool(t[1]), "trial_ms_per_substep": {k: v for k, v in ms.items() if v > 0},
            "launches_per_substep": int(t[4])}


def run_frames(solver, scen, frames, blocking):
    """Advance `frames` frames; pins and colliders re-posed before every substep.  Blocking:
    the reference ABI call by call; otherwise one xpbd_b200_step_substeps call per frame."""
    for _ in range(frames):
        if not blocking:
            scen.advance_async(solver, SUBSTEPS)
            continue
        for _ in range(SUBSTEPS):
            t = (scen.k + 1) / scen.substeps
            types, poses, dims = scen.colliders(t)
            solver.set_colliders(types, poses, dims, 0.0, 0.0)
            if scen.k > 0 and scen.has_pins():         # pins need one step first (xpbd_capi.cu:169)
                idx, pos = scen.pins(t)
                solver.set_attached(idx, pos, 1.0)
            if blocking:
                solver.step()
            else:
                solver.lib.xpbd_b200_step_async(1)
            scen.k += 1


def algorithmic_bytes(stage, sizes, n):
    """Bytes one launch of `stage` must move, counting each array of the data model once
    (FP32/int32): the per-Gaussian figures of the measurement plan."""
    m_dir = sizes[1] / n           # mean directed degree
    members = sizes[2] / n         # mean cluster members (leader excluded)
    rev = sizes[3] / n             # mean reverse-list length
    per = {
        "distance": 28 + 20 * m_dir,
        "volume_solve": 4 * members + 44,   # 36-byte cluster records
        "volume_gather": 4 * rev + 68,
        "shape": 48 + 4 * m_dir + 32,   # + the warm-start eigenvector frame, read and written
        "project": 28,
        "predict": 52,
        "velocity": 48,
    }.get(stage)
    return None if per is None else per * n


def workload_config(name, n, scen, edges_directed, members, hash_table, world):
    """The line's `config`, the same for both arms of the single-scene workloads."""
    return {"workload": name, "n_gaussians": n, "substeps_per_step": SUBSTEPS, "iterations": scen.iters,
            "graph_edges_directed": edges_directed, "cluster_members": members, "hash_table": hash_table,
            "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (working set > 2 GB per replica)"}


def max_over_ranks(values, world, device):
    """Element-wise maximum of `values` over all ranks (the job's time is its slowest rank's)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def bench_b200(args, rank, world):
    import torch

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    name, make = workload(args.config, args.gaussians)
    scen = make()
    n = scen.n
    x = pkg.XPBD()
    bind_ext(x.lib)
    stream = torch.cuda.Stream()
    x.lib.xpbd_b200_set_stream(ctypes.c_void_p(stream.cuda_stream))
    # the autotuner picks the step form (same results); a profiler's serialised launches
    # distort its trial timings, so captures fix the form with --form sequence
    x.lib.xpbd_b200_set_fused(2 if args.form == "auto" else 0)
    scen.setup(x)
    t_up = time.perf_counter()
    run_frames(x, scen, 1, blocking=True)            # upload + build (not timed)
    first_frame_s = time.perf_counter() - t_up
    bms = np.zeros(8, np.float32)
    x.lib.xpbd_b200_debug_float.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
    x.lib.xpbd_b200_debug_float(b"build_ms", bms.ctypes.data, 8)
    upload = {k: round(float(v), 1) for k, v in zip(("graph", "order", "state", "cluster_members", "cluster_lists",
                                                      "sorted_lists", "rest_state", "other"), bms)}
    upload["total"] = round(float(bms.sum()), 1)
    upload["first_frame_s"] = round(first_frame_s, 2)
    with torch.cuda.stream(stream):
        run_frames(x, scen, args.warmup, blocking=False)
        torch.cuda.synchronize()
        sizes = np.zeros(10, np.int64)
        x.lib.xpbd_b200_sizes(sizes.ctypes.data)

        # ---- timed region: device-resident throughput, one CUDA-graph replay per substep ----
        launches0 = x.lib.xpbd_b200_launch_count()
        clocks = Clocks(torch.cuda.current_device())
        clocks.start()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        run_frames(x, scen, args.steps, blocking=False)
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        clk = clocks.stop()
        ms = ev0.elapsed_time(ev1)
        launches = x.lib.xpbd_b200_launch_count() - launches0
        tuned = tuning(x.lib)

        # ---- the same frames again with a CUDA event pair around every kernel (eager
        # launches): per-stage times and the dominant kernel's mean launch duration ----
        x.lib.xpbd_b200_reset_stage_times()
        x.lib.xpbd_b200_set_profiling(1)
        run_frames(x, scen, args.steps, blocking=False)
        torch.cuda.synchronize()
        x.lib.xpbd_b200_set_profiling(0)
        st_ms = np.zeros(16)
        st_cnt = np.zeros(16, np.int64)
        k = x.lib.xpbd_b200_stage_times(st_ms.ctypes.data, st_cnt.ctypes.data, 16)
        stages = {x.lib.xpbd_b200_stage_name(s).decode(): (float(st_ms[s]), int(st_cnt[s])) for s in range(k)
                  if st_cnt[s]}

    # ---- e2e: reference ABI, host buffers, blocking step, positions read per frame ----
    x.lib.xpbd_b200_set_stream(None)
    e2e_frames = max(1, min(args.steps, 5))
    pos_bytes = n * 3 * 4
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_frames):
        run_frames(x, scen, 1, blocking=True)
        x.positions()
    e2e_s = time.perf_counter() - t0
    h2d = SUBSTEPS * (len(scen.pins(0.0)[0]) * 16 + len(scen.grippers) * 64)

    ms, e2e_ms = max_over_ranks([ms, e2e_s * 1e3], world, "cuda")
    if rank != 0:
        x.destroy()
        return None

    units = n * SUBSTEPS * args.steps * world
    value = units / (ms / 1e3)
    # the dominant single-kernel stage (the self-collision build is a chain of seven
    # short kernels: sort passes and the list build; its time is in stages_ms_per_step)
    dom = max(((k2, v) for k2, v in stages.items() if algorithmic_bytes(k2, sizes, n)), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_cnt) = dom
    peak, peak_kind = peaks()
    algo = algorithmic_bytes(dom_name, sizes, n)
    achieved = (algo / (dom_ms / dom_cnt / 1e3) / 1e9) if algo else None
    traffic = traffic_estimate(dom_name, n)
    line = {
        "metric": metric_for(args.config, n), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid scene; no public dataset)",
        "config": workload_config(name, n, scen, int(sizes[1]), int(sizes[2]), int(sizes[8]), world),
        "e2e": {"value": n * SUBSTEPS * e2e_frames * world / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": pos_bytes, "frames": e2e_frames},
        "gpu_launches": int(launches),
        "upload_ms": upload,
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo,
                     "mean_launch_ms": dom_ms / dom_cnt,
                     "measured_over": "the timed frames repeated with an event pair around each kernel"},
        "stages_ms_per_step": {k2: v[0] / args.steps for k2, v in sorted(stages.items(), key=lambda kv: -kv[1][0])},
        "clocks": clk,
        "autotuner": tuned,
    }
    line["residuals_fp64"] = residuals_fp64(x, scen)
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, scen_maker=make)
    x.destroy()
    if world == 1 and args.config == "large" and not args.no_extras:
        # the other halves of the headline metric, and the reference's own CUDA solver on
        # this workload and GPU, each at a reduced step count
        line["reference_gpu"] = reference_gpu(make, ms / (SUBSTEPS * args.steps))
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = 2, 1
        b = bench_batched(sub, 0, 1)
        line["batched"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "steps", "config", "plain",
                                             "speedup_vs_plain")}
        sv = bench_served(sub, 0, 1, duration=10.0, max_wall=20.0)
        line["served"] = {"value": sv["value"], "unit": sv["unit"], "p50_ms": sv["served"]["p50_ms"],
                          "p99_ms": sv["served"]["p99_ms"], "config": sv["config"], "served": sv["served"],
                          "served_hbm_bound": sv["served_hbm_bound"], "plain": sv["plain"],
                          "plain_engine_per_session": sv["plain_engine_per_session"],
                          "admission_target_ms": sv["admission_target_ms"],
                          "speedup_vs_plain": sv["speedup_vs_plain"],
                          "speedup_vs_plain_engine_per_session": sv["speedup_vs_plain_engine_per_session"]}
    return line


REF_SO = os.path.join(ROOT, "oracle", "_ref", "libxpbd_ref.so")


def reference_gpu(make, our_ms_per_substep, substeps=20):
    """The reference's own CUDA solver, compiled from its sources (oracle/_ref, built by
    `make -C oracle ref`), on the same workload and GPU through its C ABI: blocking
    xpbd_step per substep with pins and collider poses re-sent, as a caller does.  A
    side-by-side figure; nothing of it is on this library's path."""
    if not os.path.isfile(REF_SO):
        return {"unavailable": "oracle/_ref/libxpbd_ref.so not built (reference checkout absent at build time)"}
    scen = make()
    ref = pkg.bridge.XPBD(REF_SO)
    scen.setup(ref)
    ref.volume_stats(False)
    scen.advance(ref, 11)                        # upload, topology build, warm-up
    t0 = time.perf_counter()
    scen.advance(ref, substeps)
    dt = time.perf_counter() - t0
    ref.destroy()
    ms = dt / substeps * 1e3
    return {"impl": "reference CUDA solver compiled from its sources (sm_100a), blocking xpbd_step",
            "ms_per_substep": ms, "value": scen.n * substeps / dt, "unit": UNIT, "substeps": substeps,
            "this_ms_per_substep": our_ms_per_substep, "speedup": ms / our_ms_per_substep}


def metric_for(config, n):
    if config == "large" and n == 1_000_000:
        return METRIC
    what = {"dense": "dense contact, 20 iterations", "plain": "plain scene"}.get(config, config)
    return f"XPBD substeps/s at {n} Gaussians, {what} (Gaussian-substeps/s)"


def residuals_fp64(x, scen):
    """Constraint residuals of the final state evaluated in FP64 on the host: relative
    distance error |l - l0| / l0 over every edge, and the volume ratio J over every
    cluster (the reference's volume statistics, one more substep with them on)."""
    pos = x.positions().astype(np.float64)
    e = scen.scene["edges"]
    rest = scen.scene["rest"].astype(np.float64)
    ln = np.linalg.norm(pos[e[:, 0]] - pos[e[:, 1]], axis=1)
    rel = np.abs(ln - rest) / np.maximum(rest, 1e-12)
    x.volume_stats(True)
    run_frames_substeps(x, scen, 1)
    jm, js = x.volume_stats(True)
    x.volume_stats(False)
    return {"distance_rel_mean": float(rel.mean()), "distance_rel_p99": float(np.percentile(rel, 99)),
            "distance_rel_max": float(rel.max()), "volume_J_mean": float(jm), "volume_J_std": float(js),
            "note": "FP32 solver state, residuals in FP64"}


def run_frames_substeps(solver, scen, count):
    for _ in range(count):
        t = (scen.k + 1) / scen.substeps
        types, poses, dims = scen.colliders(t)
        solver.set_colliders(types, poses, dims, 0.0, 0.0)
        if scen.has_pins():
            idx, pos = scen.pins(t)
            solver.set_attached(idx, pos, 1.0)
        solver.step()
        scen.k += 1


def traffic_estimate(stage, n):
    """DRAM bytes per launch from the committed ncu summary of this kernel, scaled to n."""
    path = os.path.join(ROOT, "profiles", "dram_per_gaussian.json")
    if not os.path.isfile(path):
        return None
    with open(path) as f:
        d = json.load(f)
    per = d.get(stage)
    return None if per is None else per * n


def cpu_baseline(args, scen_maker, substeps=None):
    """The oracle on the host cores: the same workload, a bounded number of substeps."""
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.isfile(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    o = pkg.bridge.XPBD(lib)
    o.lib.oracle_get_threads.restype = ctypes.c_int
    scen = scen_maker()
    scen.setup(o)
    scen.advance(o, 1)                          # build (not timed)
    k = substeps or args.cpu_substeps
    t0 = time.perf_counter()
    scen.advance(o, k)
    dt = time.perf_counter() - t0
    cores = int(o.lib.oracle_get_threads())
    o.destroy()
    return {"value": scen.n * k / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{k} substeps of the same {scen.n}-Gaussian workload after its upload"}


def bench_batched(args, rank, world):
    """64 independent objects (Gaussian counts log-uniform in [2e3, 2e5]) advanced together
    as one packed scene, against the same objects stepped one at a time."""
    import torch

    batch = pkg.batch
    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    all_objs = batch.make_objects(64, seed=0)
    total = sum(sc["pos"].shape[0] for sc, _ in all_objs)
    mine = batch.partition(all_objs, world)[rank]          # this rank's objects (no exchange)
    objs = [all_objs[k] for k in mine]
    x = pkg.XPBD()
    bind_ext(x.lib)
    b = batch.Batch(objs)
    b.setup(x)
    b.advance(x, SUBSTEPS * (1 + args.warmup))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    b.advance(x, SUBSTEPS * args.steps, blocking=False)
    x.lib.xpbd_b200_sync()
    batched_s = time.perf_counter() - t0
    plain_s = 0.0
    for sc, grs in objs:
        s = batch.ObjectScenario(sc, grs)
        s.setup(x)
        s.advance(x, SUBSTEPS * (1 + args.warmup))
        x.lib.xpbd_b200_sync()
        t1 = time.perf_counter()
        s.advance(x, SUBSTEPS * args.steps)
        plain_s += time.perf_counter() - t1
    x.destroy()
    batched_s, plain_s = max_over_ranks([batched_s, plain_s], world, "cuda")
    if rank != 0:
        return None
    units = total * SUBSTEPS * args.steps
    return {"metric": "batched XPBD Gaussian-substeps/s (64 objects)", "value": units / batched_s, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batched_s / args.steps * 1e3,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (64 seeded ellipsoid objects)",
            "config": {"workload": f"batched: 64 objects, {total} Gaussians, 10 substeps x 4 iterations",
                       "objects": 64, "n_gaussians": total,
                       "parallelism": f"objects bin-packed over {world} GPU(s), no exchange"},
            "plain": {"value": units / plain_s, "unit": UNIT, "ms_per_step": plain_s / args.steps * 1e3,
                      "form": "the same objects stepped one at a time, one scene per engine"},
            "speedup_vs_plain": plain_s / batched_s}


def chainmail_seeds(scen_pos, k):
    """Step k's seeds: the 30 Gaussians nearest one x end (alternating), pushed inward by
    about one graph spacing."""
    side = -1.0 if k % 2 == 0 else 1.0
    d = np.linalg.norm(scen_pos - np.array([0.9 * side, 0.0, 0.0]), axis=1)
    idx = np.argpartition(d, 30)[:30].astype(np.int32)
    delta = np.tile(np.float32([-0.005 * side, 0.0, 0.0]), (30, 1))
    return idx, delta


def bench_chainmail(args, rank, world):
    """ChainMail on the large scene: one step = seeds + one run of the reference's default
    sweeps (20 propagation + 5 relax + 1 closing relax, forward.cu:60-64, 12808-13006)."""
    import torch

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    n = args.gaussians or 1_000_000
    sc = scenes.chainmail_scene(n, 0)
    pos64 = sc["pos"].astype(np.float64)
    x = pkg.XPBD()
    bind_ext(x.lib)
    L = x.lib
    stream = torch.cuda.Stream()
    L.xpbd_b200_set_stream(ctypes.c_void_p(stream.cuda_stream))
    x.create(sc)
    x.step()
    x.reset()
    cm = scenes.CHAINMAIL_DEFAULTS
    sweeps = cm["prop_iters"] + cm["relax_iters"] + 1
    seeds = [chainmail_seeds(pos64, k) for k in range(args.warmup + args.steps)]
    for k in range(args.warmup):
        x.chainmail_seed(*seeds[k])
        x.chainmail_run(**cm)
    launches0 = L.xpbd_b200_launch_count()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.warmup, args.warmup + args.steps):
        x.chainmail_seed(*seeds[k])
        x.chainmail_run(**cm)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = L.xpbd_b200_launch_count() - launches0
    # the dense relax sweep alone (the dominant kernel): 1 + r sweeps per call
    r = 20
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    x.chainmail_run(0, r - 1, 0.5, 0.99, 0.1)
    ev3.record(stream)
    torch.cuda.synchronize()
    relax_ms = ev2.elapsed_time(ev3) / r
    sizes = np.zeros(10, np.int64)
    L.xpbd_b200_sizes(sizes.ctypes.data)
    d = sizes[1] / n
    relax_bytes = (44 + 12 * d) * n          # pos in/out, (time, density), row offsets; nbr, rest, stiffness per edge
    peak, peak_kind = peaks()
    achieved = relax_bytes / (relax_ms / 1e3) / 1e9
    # e2e: blocking C ABI on the library's own stream, seeds from host, positions read back per step
    L.xpbd_b200_set_stream(None)
    e2e_steps = min(args.steps, 5)
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        x.chainmail_seed(*seeds[k])
        x.chainmail_run(**cm)
        x.positions()
    e2e_s = time.perf_counter() - t0
    x.destroy()
    unit = "Gaussian-sweeps/s"
    line = {
        "metric": "ChainMail Gaussian-sweeps/s at 1M Gaussians", "value": n * sweeps * args.steps / (ms / 1e3),
        "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ellipsoid scene, opacity uniform in [0.02, 1))",
        "config": {"workload": f"chainmail: {n} Gaussians, 30 seeds per step, 20 propagation + 6 relax sweeps",
                   "n_gaussians": n, "sweeps_per_step": sweeps, "l2": "inputs larger than L2"},
        "e2e": {"value": n * sweeps * e2e_steps / e2e_s, "unit": unit, "h2d_bytes_per_step": 30 * 16,
                "d2h_bytes_per_step": n * 12, "steps": e2e_steps},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "chainmail_relax", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": relax_bytes, "mean_launch_ms": relax_ms},
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        lib = os.path.join(ROOT, "oracle", "liboracle.so")
        o = pkg.bridge.XPBD(lib)
        o.CHAINMAIL_PREFIX = "oracle_"           # the oracle's ChainMail entry points
        o.lib.oracle_get_threads.restype = ctypes.c_int
        o.create(sc)
        o.step()
        o.reset()
        k = 2
        t1 = time.perf_counter()
        for j in range(k):
            o.chainmail_seed(*seeds[j])
            o.chainmail_run(**cm)
        dt = time.perf_counter() - t1
        line["cpu_baseline"] = {"value": n * sweeps * k / dt, "unit": unit, "cores": int(o.lib.oracle_get_threads()),
                                "kind": "port", "sample": f"{k} steps of the same {n}-Gaussian workload"}
        o.destroy()
    if not args.no_extras:
        line["reference_gpu"] = reference_gpu_chainmail(sc, seeds, ms / args.steps)
    return line


def reference_gpu_chainmail(sc, seeds, our_ms_per_step):
    """runChainmailGPU's dense path (forward.cu:12808-13006) of the reference compiled
    from its sources, on the same scene, seeds and sweeps, through the accessor shim."""
    if not os.path.isfile(REF_SO):
        return {"unavailable": "oracle/_ref/libxpbd_ref.so not built (reference checkout absent at build time)"}
    ref = pkg.bridge.XPBD(REF_SO)
    ref.CHAINMAIL_PREFIX = "refshim_"
    ref.create(sc)
    ref.step()
    ref.reset()
    cm = scenes.CHAINMAIL_DEFAULTS
    for k in range(2):
        ref.chainmail_seed(*seeds[k])
        ref.chainmail_run(**cm)
    steps = min(len(seeds), 5)
    t0 = time.perf_counter()
    for k in range(steps):
        ref.chainmail_seed(*seeds[k])
        ref.chainmail_run(**cm)
    dt = time.perf_counter() - t0
    ref.destroy()
    return {"impl": "reference runChainmailGPU compiled from its sources (sm_100a)", "ms_per_step": dt / steps * 1e3,
            "steps": steps, "this_ms_per_step": our_ms_per_step, "speedup": dt / steps * 1e3 / our_ms_per_step}


RENDER_W, RENDER_H, RENDER_SH = 1920, 1080, 3


def render_inputs(n):
    """The splatting workload: the large scene after 5 solver frames (grippers pulling
    and twisting), SH degree-3 colours, a camera framing the object at 1920x1080."""
    scen = scenes.large_scene_scenario(n, 0)
    colors = pkg.splat.synthetic_colors(n, RENDER_SH, 1)
    return scen, colors


def oracle_render_fn():
    lib_path = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.isfile(lib_path):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    f = ctypes.CDLL(lib_path).oracle_render
    P = ctypes.c_void_p
    f.argtypes = ([ctypes.c_int] + [P] * 5 + [ctypes.c_int] + [P] * 3 + [ctypes.c_int, ctypes.c_int]
                  + [ctypes.c_float] * 3 + [ctypes.c_int] + [P] * 3 + [ctypes.c_int] + [P] * 6)
    f.restype = ctypes.c_longlong
    return f


def oracle_render_sample(pos, sc, q, op, colors, cam):
    """One frame of the CPU restatement (single thread); returns seconds."""
    f = oracle_render_fn()
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (pos, sc, q, op, colors)]
    out = np.empty((3, cam.height, cam.width), np.float32)
    t0 = time.perf_counter()
    f(len(pos), *[v.ctypes.data for v in a], RENDER_SH, cam.view.ctypes.data, cam.proj.ctypes.data,
      cam.campos.ctypes.data, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, 1.0, 0, None, None, None, 0, None,
      out.ctypes.data, None, None, None, None)
    return time.perf_counter() - t0


def bench_render(args, rank, world):
    """Splatting (xpbd_b200_render): one step = one 1920x1080 frame of the deformed
    Gaussians (1-ring deformation fit, EWA projection, depth + tile binning, tile
    compositing), image left in device memory."""
    import torch

    torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
    n = args.gaussians or 1_000_000
    scen, colors = render_inputs(n)
    x = pkg.XPBD()
    bind_ext(x.lib)
    L = x.lib
    stream = torch.cuda.Stream()
    L.xpbd_b200_set_stream(ctypes.c_void_p(stream.cuda_stream))
    scen.setup(x)
    scen.advance(x, 5)
    pos = x.positions()
    x.render_set_colors(colors, RENDER_SH)
    x.render_set_options()
    x.render_set_floor(False)
    cam = pkg.splat.Camera.framing(pos, RENDER_W, RENDER_H)
    eps = 1e-2
    for _ in range(args.warmup):
        x.render(cam, deform_eps=eps, to_host=False)
    launches0 = L.xpbd_b200_launch_count()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        _, pairs = x.render(cam, deform_eps=eps, to_host=False)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    launches = L.xpbd_b200_launch_count() - launches0
    # stage times: the same frames with an event pair around each stage
    L.xpbd_b200_set_profiling(1)
    L.xpbd_b200_reset_stage_times()
    for _ in range(args.steps):
        x.render(cam, deform_eps=eps, to_host=False)
    st_ms, st_cnt = np.zeros(16), np.zeros(16, np.int64)
    k = L.xpbd_b200_stage_times(st_ms.ctypes.data, st_cnt.ctypes.data, 16)
    stages = {L.xpbd_b200_stage_name(i).decode(): st_ms[i] / args.steps for i in range(k) if st_cnt[i]}
    L.xpbd_b200_set_profiling(0)
    visible = int((x.render_aux(RENDER_W, RENDER_H)[3] > 0).sum())
    # the tile compositing kernel: per launch it reads each pair's index, centre, conic
    # and colour (4 + 8 + 16 + 16 B) and the tile ranges, and writes 3 colour planes,
    # transmittance and contributor count per pixel (20 B)
    npix = RENDER_W * RENDER_H
    tiles_bytes = pairs * 44 + npix * 20 + 8 * ((RENDER_W + 15) // 16) * ((RENDER_H + 15) // 16)
    tiles_ms = stages.get("render_tiles", float("nan"))
    peak, peak_kind = peaks()
    achieved = tiles_bytes / (tiles_ms / 1e3) / 1e9
    # e2e: blocking C ABI, the image read back to host memory every frame
    L.xpbd_b200_set_stream(None)
    e2e_steps = min(args.steps, 10)
    x.render(cam, deform_eps=eps, to_host=True)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        x.render(cam, deform_eps=eps, to_host=True)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    sc, q, _ = x.shapes(eps)
    op = np.asarray(scen.scene["opacity"], np.float32)
    x.destroy()
    unit = "frames/s"
    line = {
        "metric": "splatted frames/s of 1M deformed Gaussians at 1920x1080 (SH degree 3)", "value": 1e3 / ms,
        "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ellipsoid scene after 5 solver frames, seeded SH coefficients)",
        "config": {"workload": f"render: {n} Gaussians, {RENDER_W}x{RENDER_H}, SH degree {RENDER_SH}, "
                               f"deformed shapes (deform_eps {eps})",
                   "n_gaussians": n, "visible": visible, "pairs": int(pairs),
                   "l2": "inputs larger than L2 (1M Gaussians x 300 B + 13M pairs)"},
        "stages_ms": stages,
        "e2e": {"value": 1.0 / e2e_s, "unit": unit, "h2d_bytes_per_step": 4 * 35,
                "d2h_bytes_per_step": 12 * npix, "steps": e2e_steps},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "splat_tiles", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": tiles_bytes, "mean_launch_ms": tiles_ms,
                     "note": "compositing is bound by the per pixel-Gaussian exp/FMA work, not by DRAM"},
        "clocks": clk,
    }
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libxpbd_ref.so")
    if os.path.isfile(ref_so):
        f = ctypes.CDLL(ref_so).refshim_render_timed
        P = ctypes.c_void_p
        f.argtypes = ([ctypes.c_int] + [P] * 5 + [ctypes.c_int] + [P] * 3 + [ctypes.c_int, ctypes.c_int]
                      + [ctypes.c_float] * 2 + [ctypes.c_int, P])
        f.restype = ctypes.c_longlong
        out = ctypes.c_float(0.0)
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (pos, sc, q, op, colors)]
        m_ref = f(n, *[v.ctypes.data for v in a], RENDER_SH, cam.view.ctypes.data, cam.proj.ctypes.data,
                  cam.campos.ctypes.data, RENDER_W, RENDER_H, cam.tan_fovx, cam.tan_fovy, args.steps,
                  ctypes.byref(out))
        line["reference_gpu"] = {"ms_per_frame": out.value, "pairs": int(m_ref), "speedup": out.value / ms,
                                 "form": "the reference's preprocessCUDA + renderCUDA with cub scan / radix sort "
                                         "binning on the same inputs (shapes given, no physics)"}
    if not args.no_cpu_baseline:
        cs = pkg.splat.Camera.framing(pos, RENDER_W // 4, RENDER_H // 4)
        dt = oracle_render_sample(pos, sc, q, op, colors, cs)
        line["cpu_baseline"] = {"value": 1.0 / dt, "unit": unit, "cores": 1, "kind": "port",
                                "sample": f"one {cs.width}x{cs.height} frame of the same {n} Gaussians "
                                          "(a quarter of the width and height)"}
    return line


def bench_served(args, rank, world, duration=None, max_wall=None):
    """Poisson session arrivals at 200/s (5e3-5e5 Gaussians, 1-120 frames of 10 substeps x
    4 iterations) served with continuous batching in one arena, against one session at a
    time.  Sessions are admitted by the 150 GB HBM budget and, in the latency-bound run,
    also while the arena's predicted tick stays within 60 % of a 60 Hz frame (10 ms: the
    rest of the frame absorbs admission copies and host work, so that step latencies
    stay within the frame); the others wait in arrival order.  Scenes come from a pool of 12 pre-generated sizes
    (generation is host Python and would otherwise bound the arrival rate)."""
    serve = pkg.serve
    rate = 200.0
    duration = duration or 60.0
    max_wall = max_wall or (duration + 30.0)
    all_sessions = serve.make_sessions(rate, duration, seed=0, n_min=5000, n_max=500000, max_frames=120)
    if world > 1:                 # sessions bin-packed over the ranks, one arena each, no exchange
        import torch
        torch.cuda.set_device(rank % max(torch.cuda.device_count(), 1))
        mine = serve.partition_sessions(all_sessions, world)[rank]
        sessions = [all_sessions[k] for k in mine]
    else:
        sessions = all_sessions
    lib = pkg.library_path()
    t0 = time.perf_counter()
    pool = serve.scene_pool(5000, 500000, 12)
    pool.prepare_all(lib)            # each pool scene's topology, built once before the runs
    prep_s = time.perf_counter() - t0
    runs = {}
    for name, target in (("latency_bound", 0.6 * 1000.0 / 60.0), ("hbm_bound", None)):
        r = serve.run_served(lib, sessions, budget_bytes=150e9, max_wall=max_wall, latency_target_ms=target,
                             keep_results=False, pool=pool)
        r.pop("sessions_done", None)
        runs[name] = r
    plain = serve.run_plain(lib, sessions, max_wall=max_wall, pool=pool) if world == 1 else None
    # the reference runtime's pattern: an engine of its own per session (upload and
    # topology build included), one session at a time
    plain_own = serve.run_plain(lib, sessions, max_wall=max_wall, pool=list(pool)) if world == 1 else None
    pool.close()
    if world > 1:
        # whole-job figures: work summed, wall time the slowest rank's; latencies of rank 0
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, {k: (v["gauss_substeps_per_s"] * v["wall_s"], v["wall_s"]) for k, v in runs.items()})
        if rank != 0:
            return None
        for k in runs:
            work = sum(p[k][0] for p in parts)
            wall = max(p[k][1] for p in parts)
            runs[k]["gauss_substeps_per_s"] = work / wall
            runs[k]["latencies_of"] = "rank 0"
        plain = {"gauss_substeps_per_s": float("nan"), "note": "the plain loop runs at one GPU only"}
    lb = runs["latency_bound"]
    return {"metric": "served XPBD Gaussian-substeps/s with p50/p99 step latency", "value": lb["gauss_substeps_per_s"],
            "unit": UNIT, "n_gpus": world, "steps": lb["steps"], "warmup": 0,
            "ms_per_step": lb["p50_ms"], "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sessions, scenes from a pool of 12 sizes)",
            "config": {"workload": f"served: Poisson {rate:.0f}/s for {duration:.0f} s, sessions of 5e3-5e5 Gaussians, "
                                   "1-120 frames of 10 substeps x 4 iterations, HBM budget 150 GB",
                       "sessions_arrived": len(sessions), "wall_limit_s": max_wall,
                       "payloads": f"scene pool of 12 log-spaced sizes, generated and prepared at rest (topology "
                                   f"built once per pool scene) before the runs ({prep_s:.1f} s); admission = a device "
                                   "copy of the pool scene's prepared engine into the arena; the plain loop steps the "
                                   "same prepared engines, reset to rest per session"},
            "admission_target_ms": 0.6 * 1000.0 / 60.0,
            "served": lb, "served_hbm_bound": runs["hbm_bound"], "plain": plain,
            "plain_engine_per_session": plain_own,
            "speedup_vs_plain": (lb["gauss_substeps_per_s"] / max(plain["gauss_substeps_per_s"], 1e-9)
                                 if world == 1 else None),
            "speedup_vs_plain_engine_per_session": (lb["gauss_substeps_per_s"] /
                                                    max(plain_own["gauss_substeps_per_s"], 1e-9)
                                                    if world == 1 else None)}


def bench_reference(args, rank, world):
    if rank != 0:
        return None
    if args.config == "render":
        return bench_reference_render(args)
    name, make = workload(args.config, args.gaussians)
    steps = args.steps
    warm = args.warmup
    lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.isfile(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    o = pkg.bridge.XPBD(lib)
    o.lib.oracle_get_threads.restype = ctypes.c_int
    scen = make()
    scen.setup(o)
    scen.advance(o, 1 + min(warm, 1))
    t0 = time.perf_counter()
    scen.advance(o, steps)
    dt = time.perf_counter() - t0
    cores = int(o.lib.oracle_get_threads())
    value = scen.n * steps / dt
    n = scen.n
    f = o.lib.oracle_int
    f.argtypes, f.restype = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong], ctypes.c_int
    cnt = np.zeros(max(f(b"vol_count", None, 0), 1), np.int32)
    f(b"vol_count", cnt.ctypes.data, cnt.size)
    members = int(cnt.astype(np.int64).sum())
    table = 1024
    while table < 2 * n:
        table <<= 1
    cfg = workload_config(name, n, scen, 2 * len(scen.scene["edges"]), members, table if scen.self_collision else 0,
                          world)
    o.destroy()
    return {"impl": "reference", "metric": metric_for(args.config, n), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid scene; no public dataset)", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{steps} substeps (one per step) of the {n}-Gaussian workload"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def bench_reference_render(args):
    """CPU arm of the render config: the restatement (the reference has no CPU
    rasteriser), one 480x270 frame of the same Gaussians per step."""
    n = args.gaussians or 1_000_000
    scen, colors = render_inputs(n)
    sc = scen.scene
    cam = pkg.splat.Camera.framing(sc["pos"], RENDER_W // 4, RENDER_H // 4)
    steps = max(1, min(args.steps, 3))
    total = sum(oracle_render_sample(sc["pos"], sc["scales"], sc["rots"], sc["opacity"], colors, cam)
                for _ in range(steps))
    value = steps / total
    return {"impl": "reference", "metric": "splatted frames/s of 1M deformed Gaussians at 1920x1080 (SH degree 3)",
            "value": value, "unit": "frames/s", "n_gpus": 1, "steps": steps, "warmup": 0,
            "ms_per_step": total / steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded ellipsoid scene, created shapes)",
            "config": {"workload": f"render: {n} Gaussians, {cam.width}x{cam.height} CPU sample"},
            "cpu_baseline": {"value": value, "unit": "frames/s", "cores": 1, "kind": "port",
                             "sample": f"{steps} frames at {cam.width}x{cam.height}"},
            "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="large", choices=["large", "plain", "batched", "served", "chainmail", "dense", "render"])
    ap.add_argument("--cpu-substeps", type=int, default=2)
    ap.add_argument("--form", default="auto", choices=["auto", "sequence"],
                    help="step form: the autotuner's choice, or the kernel sequence (for profiler captures)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="large config: skip the batched / served / reference-GPU sub-records")
    ap.add_argument("--gaussians", type=int, default=None,
                    help="scene size of the large/plain workload (default 1,000,000 / 20,000)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "b200":
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() and args.impl == "b200" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", rank)))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            line = bench_reference(args, rank, world)
        elif args.config == "batched":
            line = bench_batched(args, rank, world)
        elif args.config == "served":
            line = bench_served(args, rank, world)
        elif args.config == "chainmail":
            line = bench_chainmail(args, rank, world)
        elif args.config == "render":
            line = bench_render(args, rank, world)
        else:
            line = bench_b200(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1 and args.impl == "b200":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
