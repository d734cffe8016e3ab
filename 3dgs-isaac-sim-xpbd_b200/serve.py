"""Continuous-batching service loop for deformation sessions.

A session is a scene plus a stream of gripper poses (frames).  Sessions arrive over
time and wait in arrival order; each is admitted while it fits the HBM budget (and, if
one is given, while the arena's predicted step time stays within a latency target).  A
session joins the serving arena (bridge.Arena) from an engine that holds its scene
prepared at rest — topology built by one upload step, then reset to the rest state
(xpbd_reset) — by a device copy of that engine's state and topology into the arena's
packed buffers, where it stays resident until its last frame.  Sessions whose scene
comes from a ScenePool share the pool scene's prepared engine (its topology is built
once); others are prepared by an admission thread on an engine of their own, beside
the GPU work of the resident sessions.  Every tick
advances every resident session by one frame with ONE library call — one launch
sequence (one CUDA-graph replay) per substep covers all of them, whatever their sizes —
carrying every session's collider poses and pin targets.  A step's latency is the time
from when it became pending (the session joined, or its previous step finished) to
when its results are ready.

The plain form for comparison steps one session at a time, start to finish, on the
same prepared engines (reset to rest before each session).
"""
import collections
import copy
import math
import queue
import threading
import time

import numpy as np

from . import bridge, scenes

BYTES_PER_GAUSSIAN = 3200   # a session engine of its own: state, graph, clusters, transposed clusters, blackboard
# arena bytes per row (Gaussian): 7 float4 state arrays, caller-order positions, order,
# object id, multiplier, rest volume terms, material, cluster record, saved inverse
# mass, three CSR row starts; per directed edge 16 B, per member and reverse entry 4 B
ARENA_ROW_BYTES = 212
ARENA_EDGES, ARENA_MEMBERS, ARENA_REV = 12, 66, 68      # capacity per row (8-NN graph, 64-member clusters)


def arena_capacity(budget_bytes):
    """(rows, edges, members, reverse entries) of an arena that fits `budget_bytes`; the
    arena's CSR offsets are 32-bit, which caps it near 31M rows at these ratios."""
    per = ARENA_ROW_BYTES + 16 * ARENA_EDGES + 4 * ARENA_MEMBERS + 4 * ARENA_REV
    rows = max(1, min(int(budget_bytes // per), (2 ** 31 - 1) // ARENA_REV))
    return rows, rows * ARENA_EDGES, rows * ARENA_MEMBERS, rows * ARENA_REV


def arena_bytes(n):
    """Arena bytes a session of n Gaussians holds (at the capacity ratios)."""
    return n * (ARENA_ROW_BYTES + 16 * ARENA_EDGES + 4 * ARENA_MEMBERS + 4 * ARENA_REV)


def make_sessions(rate, duration, seed=0, n_min=5000, n_max=500000, max_frames=120):
    """Poisson arrivals: (arrival_s, n, frames, seed) per session."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        out.append((t, n, int(rng.integers(1, max_frames + 1)), int(rng.integers(1 << 30))))
    return out


class Session:
    def __init__(self, sid, arrival, n, frames, seed, substeps=10, iters=4):
        self.sid, self.arrival, self.frames_left, self.seed = sid, arrival, frames, seed
        self.frames_total = frames
        self.substeps, self.iters = substeps, iters
        self.n = n
        self.scen = None
        self.solver = None
        self.pool_index = None
        self.src, self.own = None, False   # the engine it joins the arena from; closed after if own
        self.slot = -1
        self.final = None
        self.pending_since = None
        self.latencies = []

    def prepare(self, pool=None):
        """The session's scene and gripper stream (host work, done by the admission thread).
        With a scene `pool` (list of scenes), the pool scene closest in size stands in for
        the session's own, so that scene generation stays out of the serving loop."""
        rng = np.random.default_rng(self.seed)
        radii = tuple(float(r) for r in rng.uniform(0.3, 1.5, 3))
        if pool:
            sizes = np.array([p["pos"].shape[0] for p in pool], np.float64)
            self.pool_index = int(np.argmin(np.abs(np.log(sizes) - math.log(self.n))))
            sc = pool[self.pool_index]
            self.n = sc["pos"].shape[0]
            radii = tuple(float(v) for v in np.abs(sc["pos"]).max(0))
        else:
            sc = scenes.make_scene(self.n, self.seed, radii=radii)
        vel = (float(rng.uniform(0.002, 0.01)), 0.0, 0.0)
        twist = math.radians(float(rng.uniform(-1, 1)))
        cached = pool.grippers.get(self.pool_index) if isinstance(pool, ScenePool) else None
        if cached is None:
            g = scenes.Gripper(sc["pos"], (0.8 * radii[0], 0.0, 0.0), 20, vel, twist)
            if isinstance(pool, ScenePool):
                pool.grippers[self.pool_index] = g
        # the pinned set depends on the scene only: sessions of one pool scene share it
        g = copy.copy(pool.grippers[self.pool_index]) if isinstance(pool, ScenePool) else g
        g.velocity, g.twist = np.asarray(vel, dtype=np.float64), float(twist)
        self.scen = scenes.Scenario(sc, [g], substeps=self.substeps, iters=self.iters)

    def fresh_scenario(self):
        """A copy of the prepared scenario at frame 0 (same scene arrays)."""
        sc = self.scen
        return scenes.Scenario(sc.scene, sc.grippers, substeps=self.substeps, iters=self.iters)

    def source(self, lib_path, pool=None):
        """The engine the session joins the arena from: the pool scene's shared prepared
        engine, or (no ScenePool) one of its own, prepared here."""
        if self.scen is None:
            self.prepare(pool)
        if isinstance(pool, ScenePool) and self.pool_index is not None:
            return pool.prepared(self.pool_index, lib_path)
        self.admit(lib_path)
        return self.solver

    def admit(self, lib_path, pool=None):
        """An engine of the session's own with its scene prepared at rest."""
        if self.scen is None:
            self.prepare(pool)
        self.solver = bridge.XPBD(lib_path, instance=True)
        prepare_at_rest(self.solver, self.scen)

    def enqueue_frame(self):
        """The next frame's substeps, with their collider poses and pin targets, in one call."""
        self.scen.advance_async(self.solver, self.scen.substeps)
        self.frames_left -= 1

    def close(self, keep_result=True):
        if self.solver:
            if keep_result:
                self.final = self.solver.positions()
            self.solver.close()
            self.solver = None


def prepare_sessions(sessions, pool=None):
    """Session objects with their scenes generated, or taken from a scene pool (the
    request payloads a server receives)."""
    out = []
    for k, (a, n, frames, seed) in enumerate(sessions):
        s = Session(k, a, n, frames, seed)
        s.prepare(pool)
        out.append(s)
    return out


def partition_sessions(sessions, ranks):
    """Sessions split over `ranks` GPUs, each with an arena of its own: longest work first
    (Gaussians x frames) onto the least loaded rank, each rank's share in arrival order.
    Sessions are independent, so the ranks exchange nothing while they serve."""
    def work(item):
        return item.n * item.frames_total if isinstance(item, Session) else item[1] * item[2]
    order = sorted(range(len(sessions)), key=lambda k: (-work(sessions[k]), k))
    load = [0.0] * ranks
    bins = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda q: (load[q], q))
        bins[r].append(k)
        load[r] += work(sessions[k])
    return [sorted(b) for b in bins]


class ScenePool(list):
    """Scenes standing in for request payloads (a list of scene dicts), each with an engine
    that holds it prepared at rest, built on first use (`prepared`) or all at once
    (`prepare_all`): create, the session settings, one upload step, reset."""

    def __init__(self, items, substeps=10, iters=4):
        super().__init__(items)
        self.substeps, self.iters = substeps, iters
        self.engines = {}
        self.grippers = {}   # pool index -> gripper with the pinned set (the same for every session)

    def index_for(self, n):
        sizes = np.array([p["pos"].shape[0] for p in self], np.float64)
        return int(np.argmin(np.abs(np.log(sizes) - math.log(n))))

    def prepared(self, k, lib_path):
        eng = self.engines.get(k)
        if eng is None:
            eng = bridge.XPBD(lib_path, instance=True)
            prepare_at_rest(eng, scenes.Scenario(self[k], [], substeps=self.substeps, iters=self.iters))
            self.engines[k] = eng
        return eng

    def prepare_all(self, lib_path):
        for k in range(len(self)):
            self.prepared(k, lib_path)

    def close(self):
        for eng in self.engines.values():
            eng.close()
        self.engines = {}


def prepare_at_rest(solver, scen):
    """Settings of `scen` on `solver`, its scene uploaded and the topology built by one
    step, then the state reset to rest (positions, velocities, multipliers)."""
    scen.setup(solver)
    solver.step()
    solver.reset()
    scen.k = 0


def scene_pool(n_min, n_max, count=12, seed=0):
    """`count` scenes with log-spaced sizes in [n_min, n_max] (the config-0 distribution)."""
    sizes = np.exp(np.linspace(math.log(n_min), math.log(n_max), count))
    return ScenePool([scenes.make_scene(int(round(n)), seed + k) for k, n in enumerate(sizes)])


def _frame_arrays(resident, substeps):
    """Collider poses and pin targets of the next frame of every resident session, as
    the arena's step call takes them (a session's inputs prepared ahead, `next_inputs`,
    are used when they are for its current substep)."""
    types, poses, dims, cslot, pslot, pidx, targets = [], [], [], [], [], [], []
    for s in resident:
        pre = getattr(s, "next_inputs", None)
        ty, po, di, idx, tg = pre[1] if pre is not None and pre[0] == s.scen.k else s.scen.frame_inputs(substeps)
        types.append(ty); poses.append(po); dims.append(di); cslot.append(np.full(len(ty), s.slot, np.int32))
        pidx.append(idx); targets.append(tg); pslot.append(np.full(len(idx), s.slot, np.int32))
    cat = np.concatenate
    return (cat(types), cat(poses, axis=1), cat(dims), cat(cslot), cat(pslot), cat(pidx), cat(targets, axis=1))


def run_served(lib_path, sessions, budget_bytes=150e9, time_scale=1.0, max_wall=None, latency_target_ms=None,
               keep_results=True, pool=None):
    """Serve `sessions` (tuples from make_sessions, or prepared Session objects) with
    continuous batching in one arena.  Admission in arrival order while the session fits
    the budget and — with `latency_target_ms` — while the resident Gaussians, at the
    throughput measured so far, keep a tick within the target.  Sessions given as tuples
    are prepared when admitted (from `pool` when given).  With a ScenePool a session
    joins straight from its pool scene's prepared engine; otherwise the admission thread
    prepares an engine of its own first.  Returns stats."""
    t0 = time.perf_counter()
    arena = bridge.Arena(lib_path, *arena_capacity(budget_bytes))
    shared = isinstance(pool, ScenePool)
    arrivals = collections.deque(sessions)
    ready = queue.Queue()
    stop = threading.Event()
    backlog = queue.Queue()
    errors = []

    def admitter():
        while not stop.is_set():
            try:
                sess = backlog.get(timeout=0.05)
            except queue.Empty:
                continue
            try:
                sess.src, sess.own = sess.source(lib_path, pool), True
            except Exception as e:   # surfaced by the serving loop
                errors.append(e)
            ready.put(sess)

    worker = threading.Thread(target=admitter, daemon=True)
    worker.start()
    waiting = collections.deque()
    resident, joining = [], []
    done, work, ticks, resident_bytes, resident_gauss, queued = [], 0, 0, 0.0, 0, 0
    throughput = 2.0e8           # Gaussian-substeps/s: a prior, then the ticks' running mean
    phase = {"admit": 0.0, "inputs": 0.0, "step_call": 0.0, "prefetch": 0.0, "sync": 0.0}   # host seconds
    waits = []
    sid = 0
    try:
        while arrivals or waiting or resident or joining or queued > len(done):
            now = time.perf_counter() - t0
            if max_wall and now > max_wall:
                break
            if errors:
                raise errors[0]
            while arrivals and _arrival(arrivals[0]) * time_scale <= now:
                item = arrivals.popleft()
                if isinstance(item, Session):
                    waiting.append(item)
                else:
                    a, n, frames, seed = item
                    if pool:                 # the pool scene that will stand in for it
                        n = min((p["pos"].shape[0] for p in pool), key=lambda v: abs(math.log(v) - math.log(n)))
                    waiting.append(Session(sid, a * time_scale, n, frames, seed))
                sid += 1
            # admission in arrival order: HBM budget, then the latency target
            while waiting:
                s = waiting[0]
                need = arena_bytes(s.n)
                if resident_bytes + need > budget_bytes:
                    break
                if latency_target_ms and resident_gauss > 0:
                    tick_ms = (resident_gauss + s.n) * s.substeps / throughput * 1e3
                    if tick_ms > latency_target_ms:
                        break
                resident_bytes += need
                resident_gauss += s.n
                s = waiting.popleft()
                queued += 1
                if shared:
                    if s.scen is None:
                        s.prepare(pool)
                    s.src, s.own = s.source(lib_path, pool), False
                    ready.put(s)
                else:
                    backlog.put(s)
            while not ready.empty():
                joining.append(ready.get())
            still_joining = []
            t_adm = time.perf_counter()
            for s in joining:
                slot = arena.admit(s.src) if not still_joining else None
                if slot is None:          # full until sessions leave (compaction ran already); the
                    still_joining.append(s)   # later ones keep their arrival order behind it
                    continue
                s.slot = slot
                if s.own:                 # the arena holds the session's state now
                    s.src.close()
                    s.solver = None
                s.src = None
                s.pending_since = time.perf_counter()
                waits.append(s.pending_since - t0 - s.arrival)
                resident.append(s)
            joining = still_joining
            phase["admit"] += time.perf_counter() - t_adm
            if not resident:
                time.sleep(0.001)
                continue
            sub = resident[0].scen.substeps
            t_in = time.perf_counter()
            ty, po, di, cs, ps, pi, tg = _frame_arrays(resident, sub)
            t_tick = time.perf_counter()
            arena.step(sub, ty, po, di, cs, ps, pi, tg)
            t_call = time.perf_counter()
            # while the GPU runs this tick: the next frame's inputs of the sessions that stay
            for s in resident:
                if s.frames_left > 1:
                    s.next_inputs = (s.scen.k + sub, s.scen.frame_inputs(sub, s.scen.k + sub))
            t_pre = time.perf_counter()
            arena.sync()
            t_end = time.perf_counter()
            phase["inputs"] += t_tick - t_in
            phase["step_call"] += t_call - t_tick
            phase["prefetch"] += t_pre - t_call
            phase["sync"] += t_end - t_pre
            ticks += 1
            tick_work = sum(s.n for s in resident) * sub
            rate = tick_work / max(t_end - t_tick, 1e-9)
            throughput = 0.8 * throughput + 0.2 * rate
            still = []
            for s in resident:
                s.scen.k += sub
                s.frames_left -= 1
                s.latencies.append(t_end - s.pending_since)
                s.pending_since = t_end
                work += s.n * sub
                if s.frames_left <= 0:
                    if keep_results:
                        s.final = arena.positions(s.slot, s.n)
                    arena.retire(s.slot)
                    resident_bytes -= arena_bytes(s.n)
                    resident_gauss -= s.n
                    done.append(s)
                else:
                    still.append(s)
            resident = still
    finally:
        stop.set()
        worker.join(timeout=5)
        usage = arena.usage()
        arena.close()
    wall = time.perf_counter() - t0
    lat = np.concatenate([np.asarray(s.latencies) for s in done]) if done else np.zeros(1)
    return {"sessions": len(done), "steps": int(lat.size), "wall_s": wall, "ticks": ticks,
            "gauss_substeps_per_s": work / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "admission_wait_p50_s": float(np.percentile(waits, 50)) if waits else 0.0,
            "arena_rows_cap": usage["rows_cap"], "host_phase_s": {k: round(v, 3) for k, v in phase.items()},
            "sessions_done": done}


def _arrival(item):
    return item.arrival if isinstance(item, Session) else item[0]


def run_plain(lib_path, sessions, max_wall=None, pool=None):
    """One session at a time, start to finish (no overlap): on its pool scene's prepared
    engine, reset to rest before and after, with a ScenePool; else on an engine of its
    own."""
    t0 = time.perf_counter()
    work, lats, count = 0, [], 0
    shared = isinstance(pool, ScenePool)
    for k, item in enumerate(sessions):
        if max_wall and time.perf_counter() - t0 > max_wall:
            break
        if isinstance(item, Session):
            s = Session(item.sid, item.arrival, item.n, item.frames_total, item.seed)
            s.scen = item.fresh_scenario()
            s.pool_index = item.pool_index
        else:
            a, n, frames, seed = item
            s = Session(k, a, n, frames, seed)
        if shared:
            if s.scen is None:
                s.prepare(pool)
            s.solver = pool.prepared(s.pool_index, lib_path)
            s.solver.reset()
        else:
            s.admit(lib_path, pool)
        while s.frames_left > 0:
            t1 = time.perf_counter()
            s.enqueue_frame()
            s.solver.lib.xpbd_b200_sync()
            lats.append(time.perf_counter() - t1)
            work += s.n * s.scen.substeps
        if shared:
            s.solver.reset()
            s.solver = None
        else:
            s.close()
        count += 1
    wall = time.perf_counter() - t0
    lat = np.asarray(lats) if lats else np.zeros(1)
    return {"sessions": count, "steps": int(lat.size), "wall_s": wall, "gauss_substeps_per_s": work / wall,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
