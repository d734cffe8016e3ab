"""Continuous-batching service loop for deformation sessions.

A session is a scene plus a stream of gripper poses (frames).  Sessions arrive over
time; each is admitted while the resident solver state fits the HBM budget, uploaded
by a background admission thread (host topology build + upload run beside the GPU
work of the sessions already resident), and kept resident — one engine instance with
its own CUDA stream per session — until its last frame.  Every tick, each resident
session with a pending frame enqueues that frame's substeps on its stream; the GPU
runs all of them concurrently, and the tick ends when all are done.  A step's latency
is the time from when it became pending (its session was admitted, or its previous
step finished) to when its results are ready.

The plain form for comparison steps one session at a time, start to finish.
"""
import collections
import math
import queue
import threading
import time

import numpy as np

from . import bridge, scenes

BYTES_PER_GAUSSIAN = 3200   # resident estimate: state, graph, clusters, transposed clusters, blackboard


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
        self.pending_since = None
        self.latencies = []

    def prepare(self):
        """The session's scene and gripper stream (host work, done by the admission thread)."""
        rng = np.random.default_rng(self.seed)
        radii = tuple(float(r) for r in rng.uniform(0.3, 1.5, 3))
        sc = scenes.make_scene(self.n, self.seed, radii=radii)
        vel = (float(rng.uniform(0.002, 0.01)), 0.0, 0.0)
        g = scenes.Gripper(sc["pos"], (0.8 * radii[0], 0.0, 0.0), 20, vel, math.radians(float(rng.uniform(-1, 1))))
        self.scen = scenes.Scenario(sc, [g], substeps=self.substeps, iters=self.iters)

    def fresh_scenario(self):
        """A copy of the prepared scenario at frame 0 (same scene arrays)."""
        sc = self.scen
        return scenes.Scenario(sc.scene, sc.grippers, substeps=self.substeps, iters=self.iters)

    def admit(self, lib_path):
        if self.scen is None:
            self.prepare()
        self.solver = bridge.XPBD(lib_path, instance=True)
        self.scen.setup(self.solver)
        self.scen.advance(self.solver, 1)          # upload + topology build (first substep)

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


def prepare_sessions(sessions):
    """Session objects with their scenes generated (the request payloads a server receives)."""
    out = []
    for k, (a, n, frames, seed) in enumerate(sessions):
        s = Session(k, a, n, frames, seed)
        s.prepare()
        out.append(s)
    return out


def run_served(lib_path, sessions, budget_bytes=150e9, time_scale=1.0, max_wall=None):
    """Serve `sessions` (tuples from make_sessions, or prepared Session objects) with
    continuous batching.  Returns stats."""
    t0 = time.perf_counter()
    arrivals = collections.deque(sessions)
    ready = queue.Queue()
    resident = []
    resident_bytes = [0.0]
    lock = threading.Lock()
    stop = threading.Event()
    queued = [0]                # sessions handed to the admission thread
    backlog = queue.Queue()

    def admitter():
        while not stop.is_set():
            try:
                sess = backlog.get(timeout=0.05)
            except queue.Empty:
                continue
            sess.admit(lib_path)
            ready.put(sess)

    worker = threading.Thread(target=admitter, daemon=True)
    worker.start()
    waiting = collections.deque()
    done, work, ticks = [], 0, 0
    sid = 0
    while arrivals or waiting or resident or queued[0] > len(done):
        now = time.perf_counter() - t0
        if max_wall and now > max_wall:
            break
        while arrivals and _arrival(arrivals[0]) * time_scale <= now:
            item = arrivals.popleft()
            if isinstance(item, Session):
                waiting.append(item)
            else:
                a, n, frames, seed = item
                waiting.append(Session(sid, a * time_scale, n, frames, seed))
            sid += 1
        # admission by resident-byte budget, in arrival order
        while waiting:
            need = waiting[0].n * BYTES_PER_GAUSSIAN
            with lock:
                if resident_bytes[0] + need > budget_bytes:
                    break
                resident_bytes[0] += need
            backlog.put(waiting.popleft())
            queued[0] += 1
        while not ready.empty():
            s = ready.get()
            s.pending_since = time.perf_counter()
            resident.append(s)
        if not resident:
            time.sleep(0.001)
            continue
        for s in resident:
            s.enqueue_frame()
        for s in resident:
            s.solver.lib.xpbd_b200_sync()
        t_end = time.perf_counter()
        ticks += 1
        still = []
        for s in resident:
            s.latencies.append(t_end - s.pending_since)
            s.pending_since = t_end
            work += s.n * s.scen.substeps
            if s.frames_left <= 0:
                with lock:
                    resident_bytes[0] -= s.n * BYTES_PER_GAUSSIAN
                s.close()
                done.append(s)
            else:
                still.append(s)
        resident = still
    stop.set()
    worker.join(timeout=5)
    wall = time.perf_counter() - t0
    lat = np.concatenate([np.asarray(s.latencies) for s in done]) if done else np.zeros(1)
    return {"sessions": len(done), "steps": int(lat.size), "wall_s": wall, "ticks": ticks,
            "gauss_substeps_per_s": work / wall, "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "sessions_done": done}


def _arrival(item):
    return item.arrival if isinstance(item, Session) else item[0]


def run_plain(lib_path, sessions, max_wall=None):
    """One session at a time, start to finish, on one engine (no overlap)."""
    t0 = time.perf_counter()
    work, lats, count = 0, [], 0
    for k, item in enumerate(sessions):
        if max_wall and time.perf_counter() - t0 > max_wall:
            break
        if isinstance(item, Session):
            s = Session(item.sid, item.arrival, item.n, item.frames_total, item.seed)
            s.scen = item.fresh_scenario()
        else:
            a, n, frames, seed = item
            s = Session(k, a, n, frames, seed)
        s.admit(lib_path)
        while s.frames_left > 0:
            t1 = time.perf_counter()
            s.enqueue_frame()
            s.solver.lib.xpbd_b200_sync()
            lats.append(time.perf_counter() - t1)
            work += s.n * s.scen.substeps
        s.close()
        count += 1
    wall = time.perf_counter() - t0
    lat = np.asarray(lats) if lats else np.zeros(1)
    return {"sessions": count, "steps": int(lat.size), "wall_s": wall, "gauss_substeps_per_s": work / wall,
            "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)}
