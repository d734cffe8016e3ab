"""Batched objects: many independent objects packed into one solver scene.

Every kernel of the step works per Gaussian, per cluster or per edge of the graph, and
objects are separate graph components, so K objects concatenated into one scene are
advanced by the same launches as one object — one graph-captured kernel sequence per
substep covers them all, whatever their sizes.  Objects keep their own coordinates
(they may overlap in space); each object's grippers act only on that object
(xpbd_b200_set_colliders_many binds every collider to its object), self-collision and ground stay off, so every
object's trajectory is the one it has alone, bit for bit (tests/test_gpu_batch.py).
"""
import ctypes
import math

import numpy as np

from . import scenes


def make_objects(count=64, seed=0, n_min=2000, n_max=200000, radius_range=(0.3, 1.5)):
    """Seeded independent objects: Gaussian counts log-uniform in [n_min, n_max], each an
    ellipsoid with radii drawn in `radius_range`, and 1-2 capsule grippers at its x
    extremes moving on linear-plus-twist trajectories."""
    rng = np.random.default_rng(seed)
    objs = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        radii = tuple(float(r) for r in rng.uniform(*radius_range, 3))
        sc = scenes.make_scene(n, seed * 1000 + k + 1, radii=radii)
        ng = int(rng.integers(1, 3))
        grippers = []
        for g in range(ng):
            side = -1.0 if g == 0 else 1.0
            centre = (side * 0.8 * radii[0], 0.0, 0.0)
            vel = (side * float(rng.uniform(0.002, 0.01)), float(rng.uniform(-0.005, 0.005)), 0.0)
            twist = math.radians(float(rng.uniform(-1.0, 1.0)))
            gr = scenes.Gripper(sc["pos"], centre, 20, vel, twist)
            inside = scenes.Gripper(sc["pos"], centre, 0, vel, twist, pin_radius=0.055)
            gr.idx = np.union1d(gr.idx, inside.idx).astype(np.int32)
            gr.rel = sc["pos"][gr.idx].astype(np.float64) - gr.centre
            grippers.append(gr)
        objs.append((sc, grippers))
    return objs


def object_cost(scene, cap=64):
    """Per-step work of an object: Gaussians x (mean directed degree + cluster members)."""
    n = scene["pos"].shape[0]
    return n * (2.0 * len(scene["edges"]) / max(n, 1) + cap)


def partition(objects, ranks, cap=64):
    """Objects split over `ranks` GPUs (longest-processing-time greedy bin packing on
    object_cost): returns one list of object indices per rank, each in input order.
    Objects are independent, so the ranks share nothing during the step."""
    order = sorted(range(len(objects)), key=lambda k: (-object_cost(objects[k][0], cap), k))
    load = [0.0] * ranks
    bins = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda q: (load[q], q))
        bins[r].append(k)
        load[r] += object_cost(objects[k][0], cap)
    return [sorted(b) for b in bins]


class ObjectScenario(scenes.Scenario):
    """One object of a batch run on its own (the reference's one-scene-per-instance form)."""

    def __init__(self, scene, grippers, **kw):
        kw.setdefault("self_collision", False)
        super().__init__(scene, grippers, **kw)


class Batch(scenes.Scenario):
    """K objects concatenated into one scene; pins and colliders re-posed per substep
    like Scenario, with each collider restricted to its own object."""

    def __init__(self, objects, **kw):
        kw.setdefault("self_collision", False)
        merged = scenes.merge_scenes([sc for sc, _ in objects])
        grippers, owner = [], []
        self.offsets = [0]
        for k, (sc, grs) in enumerate(objects):
            base = self.offsets[-1]
            for g in grs:
                g2 = scenes.Gripper.__new__(scenes.Gripper)
                g2.__dict__.update(g.__dict__)
                g2.idx = (g.idx + base).astype(np.int32)
                grippers.append(g2)
                owner.append(k)
            self.offsets.append(base + sc["pos"].shape[0])
        super().__init__(merged, grippers, **kw)
        self.owner = np.asarray(owner, np.int32)
        self.objects = objects

    def colliders_posed(self, solver, t):
        types, poses, dims = self.colliders(t)
        types = np.ascontiguousarray(np.asarray(types, np.int32))
        poses = np.ascontiguousarray(np.asarray(poses, np.float32).reshape(-1))
        dims = np.ascontiguousarray(np.asarray(dims, np.float32).reshape(-1))
        L = solver.lib
        L.xpbd_b200_set_colliders_many.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_float] * 2
        rc = L.xpbd_b200_set_colliders_many(len(types), types.ctypes.data, poses.ctypes.data, dims.ctypes.data,
                                            self.owner.ctypes.data, 0.0, 0.0)
        if rc != 0:
            raise RuntimeError(solver.last_error())

    def advance(self, solver, count, blocking=True):
        for _ in range(count):
            t = (self.k + 1) / self.substeps
            self.colliders_posed(solver, t)
            if self.k > 0 and self.grippers:
                idx, pos = self.pins(t)
                solver.set_attached(idx, pos, 1.0)
            if blocking:
                solver.step()
            else:
                solver.lib.xpbd_b200_step_async(1)
            self.k += 1

    def split(self, arr):
        """Per-object views of a (N, ...) array of the merged scene."""
        return [arr[self.offsets[k]:self.offsets[k + 1]] for k in range(len(self.objects))]
