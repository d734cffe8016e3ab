"""Seeded synthetic Gaussian scenes and gripper scenarios.

The reference ships no asset (its Wolf bundle is absent, docs/data.md:3) and no
benchmark harness, so every workload here is generated: Gaussian centres uniform in
an ellipsoid, random unit quaternions (w, x, y, z), log-normal scales, a symmetric
k-NN distance graph with rest lengths taken from the initial pose, and one or two
capsule grippers that pin their nearest Gaussians and move them per substep.

The arrays match the inputs of ``xpbd_create`` (xpbd_capi.cu:71-102): ``pos[n,3]``,
``scales[n,3]`` (activated), ``rots[n,4]`` (normalised, w,x,y,z), ``opacity[n]``
(activated), undirected edges ``[e,2]`` with i<j, ``rest[e]``, ``stiff[e]``.
"""
import ctypes
import math

import numpy as np

DEFAULT_RADII = (1.0, 0.6, 0.4)


def make_scene(n, seed=0, radii=DEFAULT_RADII, knn=8, centre=(0.0, 0.0, 0.0), opacity=0.9):
    """One object: ``n`` Gaussians uniform in an ellipsoid with ``radii``.

    Edges are the symmetric union of each centre's ``knn`` nearest neighbours,
    deduplicated to i<j and sorted; rest = float32 |x_i - x_j|; stiffness 1.
    """
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    u = rng.random(n) ** (1.0 / 3.0)
    pos = (d * u[:, None] * np.asarray(radii, dtype=np.float64) + np.asarray(centre)).astype(np.float32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    scales = np.exp(rng.normal(-4.0, 0.3, (n, 3))).astype(np.float32)
    k = min(knn + 1, n)
    _, nn = cKDTree(pos.astype(np.float64)).query(pos.astype(np.float64), k=k)
    nn = nn.reshape(n, k)
    i = np.repeat(np.arange(n, dtype=np.int64), k - 1)
    j = nn[:, 1:].reshape(-1).astype(np.int64)
    a, b = np.minimum(i, j), np.maximum(i, j)
    keep = a != b
    key = np.unique(a[keep] * n + b[keep])
    edges = np.stack([key // n, key % n], axis=1).astype(np.int32)
    diff = pos[edges[:, 0]].astype(np.float64) - pos[edges[:, 1]].astype(np.float64)
    rest = np.sqrt((diff * diff).sum(1)).astype(np.float32)
    return {
        "pos": np.ascontiguousarray(pos),
        "scales": np.ascontiguousarray(scales),
        "rots": np.ascontiguousarray(q.astype(np.float32)),
        "opacity": np.full(n, opacity, dtype=np.float32),
        "edges": np.ascontiguousarray(edges),
        "rest": np.ascontiguousarray(rest),
        "stiff": np.ones(len(edges), dtype=np.float32),
    }


def merge_scenes(parts):
    """Concatenate independent objects into one scene (edges re-indexed)."""
    out = {k: [] for k in ("pos", "scales", "rots", "opacity", "edges", "rest", "stiff")}
    base = 0
    for p in parts:
        for k in ("pos", "scales", "rots", "opacity", "rest", "stiff"):
            out[k].append(p[k])
        out["edges"].append(p["edges"] + base)
        base += p["pos"].shape[0]
    return {k: np.ascontiguousarray(np.concatenate(v, axis=0)) for k, v in out.items()}


def _rot_x(angle):
    c, s = math.cos(angle), math.sin(angle)
    return np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]], dtype=np.float64)


class Gripper:
    """A capsule (radius, half-length along local z) that pins the ``count`` Gaussians
    nearest to ``centre`` (or, with ``pin_radius``, every Gaussian that close to its axis)
    and moves them rigidly: translation ``velocity`` per frame, rotation ``twist`` radians
    per frame about the world x axis through its centre."""

    def __init__(self, pos, centre, count=200, velocity=(0.01, 0.0, 0.0), twist=0.0,
                 radius=0.05, half_length=0.05, pin_radius=None):
        self.centre = np.asarray(centre, dtype=np.float64)
        p = pos.astype(np.float64) - self.centre
        if pin_radius is None:
            d2 = (p ** 2).sum(1)
            count = min(count, len(pos))
            self.idx = np.sort(np.argsort(d2, kind="stable")[:count]).astype(np.int32)
        else:
            # every Gaussian within pin_radius of the capsule's axis segment (local z)
            z = np.clip(p[:, 2], -half_length, half_length)
            d2 = p[:, 0] ** 2 + p[:, 1] ** 2 + (p[:, 2] - z) ** 2
            self.idx = np.nonzero(d2 <= pin_radius * pin_radius)[0].astype(np.int32)
        self.rel = pos[self.idx].astype(np.float64) - self.centre
        self.velocity = np.asarray(velocity, dtype=np.float64)
        self.twist = float(twist)
        self.radius = radius
        self.half_length = half_length

    def pose(self, t):
        """(R 3x3, centre 3) after ``t`` frames."""
        return _rot_x(self.twist * t), self.centre + self.velocity * t

    def targets(self, t):
        R, c = self.pose(t)
        return (c + self.rel @ R.T).astype(np.float32)

    def collider(self, t):
        R, c = self.pose(t)
        return 2, np.concatenate([R.reshape(-1), c]).astype(np.float32), \
            np.array([self.radius, self.half_length, 0.0], np.float32)


class Scenario:
    """Drives any object with the ``XPBD`` method set through ``frames`` 60 Hz frames of
    ``substeps`` solver steps each (one ``xpbd_step`` per substep, dt = 1/(60*substeps)).

    Before every substep the grippers' capsules are re-posed and their pinned Gaussians
    re-targeted by linear interpolation of the per-frame motion.  The reference rejects
    ``xpbd_set_attached`` before the first step (xpbd_capi.cu:169), so pins start with the
    second substep on every backend alike.
    """

    def __init__(self, scene, grippers, substeps=10, iters=4, shape=True, volume=True, self_collision=False,
                 within_body=True, ring_k=3, max_members=64, leader_min_hop=1, dist_compliance=1e-6,
                 vol_compliance=1e-5, shape_compliance=1e-5, under_relax=0.6, vel_damping=0.01,
                 shape_robust=True, frame_dt=1.0 / 60.0, object_shape=0.0):
        self.scene = scene
        self.object_shape = object_shape
        self.grippers = list(grippers)
        self.substeps = substeps
        self.iters = iters
        self.shape = shape
        self.volume = volume
        self.self_collision = self_collision
        self.within_body = within_body
        self.ring_k = ring_k
        self.max_members = max_members
        self.leader_min_hop = leader_min_hop
        self.dist_compliance = dist_compliance
        self.vol_compliance = vol_compliance
        self.shape_compliance = shape_compliance
        self.under_relax = under_relax
        self.vel_damping = vel_damping
        self.shape_robust = shape_robust
        self.dt = frame_dt / substeps
        self.k = 0

    @property
    def n(self):
        return self.scene["pos"].shape[0]

    def setup(self, solver):
        solver.create(self.scene)
        solver.set_solver(iters=self.iters, dt=self.dt, under_relax=self.under_relax,
                          vel_damping=self.vel_damping, dist_compliance=self.dist_compliance,
                          shape_compliance=self.shape_compliance)
        solver.set_constraints(distance=True, shape=self.shape, angle=False, volume=self.volume)
        solver.set_volume(self.vol_compliance, self.ring_k, self.max_members, self.leader_min_hop)
        solver.set_shape_robust(self.shape_robust)
        solver.set_self_collision(self.self_collision, 1.5, 2.0, self.within_body)
        solver.set_object_shape(self.object_shape)   # settings outlive create / destroy: always set
        solver.set_ground(False, (0.0, 0.0, 1.0), 0.0, gravity=0.0)
        solver.set_colliders([], [], [])   # drops the last scene's collider poses (friction velocity)
        solver.volume_stats(False)
        self.k = 0

    def has_pins(self):
        return any(len(g.idx) for g in self.grippers)

    def pins(self, t):
        if not self.grippers:
            return None, None
        idx = np.concatenate([g.idx for g in self.grippers])
        pos = np.concatenate([g.targets(t) for g in self.grippers], axis=0)
        return idx, pos

    def colliders(self, t):
        cols = [g.collider(t) for g in self.grippers]
        if not cols:
            return [], np.zeros((0, 12), np.float32), np.zeros((0, 3), np.float32)
        return [c[0] for c in cols], np.stack([c[1] for c in cols]), np.stack([c[2] for c in cols])

    def frame_inputs(self, count, k0=None):
        """The next ``count`` substeps' collider poses (count, K, 12) and pin targets
        (count, P, 3), with the collider types and dims and the pinned indices; from
        substep ``k0`` instead of the current one when given."""
        k0 = self.k if k0 is None else k0
        ts = [(k0 + 1 + s) / self.substeps for s in range(count)]
        types, _, dims = self.colliders(ts[0])
        poses = np.stack([self.colliders(t)[1] for t in ts]).astype(np.float32) if self.grippers \
            else np.zeros((count, 0, 12), np.float32)
        if self.has_pins():
            idx = np.concatenate([g.idx for g in self.grippers]).astype(np.int32)
            targets = np.stack([np.concatenate([g.targets(t) for g in self.grippers], axis=0) for t in ts])
        else:
            idx, targets = np.zeros(0, np.int32), np.zeros((count, 0, 3), np.float32)
        return (np.asarray(types, np.int32), np.ascontiguousarray(poses), np.asarray(dims, np.float32).reshape(-1, 3),
                idx, np.ascontiguousarray(targets, np.float32))

    def advance_async(self, solver, count):
        """Enqueue ``count`` substeps with one library call (xpbd_b200_step_substeps)."""
        types, poses, dims, idx, targets = self.frame_inputs(count)
        raw = getattr(solver, "raw", solver.lib).xpbd_b200_step_substeps   # the ctypes function itself
        raw.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                        ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        raw.restype = ctypes.c_int
        f = solver.lib.xpbd_b200_step_substeps   # through the engine selection of an instance
        dims = np.ascontiguousarray(dims)
        rc = f(count, len(types), types.ctypes.data, poses.ctypes.data, dims.ctypes.data, 0.0, 0.0, len(idx),
               idx.ctypes.data, targets.ctypes.data)
        if rc != 0:
            raise RuntimeError(solver.last_error())
        self.k += count

    def advance(self, solver, count):
        """Run ``count`` substeps."""
        for _ in range(count):
            t = (self.k + 1) / self.substeps
            if self.grippers:
                types, poses, dims = self.colliders(t)
                solver.set_colliders(types, poses, dims, 0.0, 0.0)
                if self.k > 0 and self.has_pins():
                    idx, pos = self.pins(t)
                    solver.set_attached(idx, pos, 1.0)
            solver.step()
            self.k += 1


def plain_scene_scenario(n=20000, seed=0, **kw):
    """The plain small-scene workload: one object, two capsule grippers at the x extremes
    (+-0.9, 0, 0), each pinning its 200 nearest Gaussians; both translate +0.01 x per frame."""
    scene = make_scene(n, seed)
    pins = kw.pop("pins", 200)
    grippers = [Gripper(scene["pos"], (-0.9, 0.0, 0.0), pins, (0.01, 0.0, 0.0)),
                Gripper(scene["pos"], (0.9, 0.0, 0.0), pins, (0.01, 0.0, 0.0))]
    return Scenario(scene, grippers, **kw)


def large_scene_scenario(n=1_000_000, seed=0, **kw):
    """The large single-scene workload: grippers pull apart (+-0.01 x per frame) while each
    twists 1 degree per frame about x; self-collision on (within-body pairs).  Each gripper
    pins every Gaussian inside its capsule (radius 0.05 + 10 %), so no free Gaussian starts
    inside a collider at any scene size."""
    scene = kw.pop("scene", None) or make_scene(n, seed)
    deg = math.radians(1.0)
    grippers = [Gripper(scene["pos"], (-0.9, 0.0, 0.0), 0, (-0.01, 0.0, 0.0), -deg, pin_radius=0.055),
                Gripper(scene["pos"], (0.9, 0.0, 0.0), 0, (0.01, 0.0, 0.0), deg, pin_radius=0.055)]
    kw.setdefault("self_collision", True)
    kw.setdefault("within_body", True)
    return Scenario(scene, grippers, **kw)


class Plate:
    """A box collider (type 1, half extents ``half``) whose inner face starts at height
    ``face`` on the ``side`` (+1 above, -1 below) of the z axis and moves toward z = 0 by
    ``speed`` per frame until it has travelled ``travel``; it pins nothing."""

    def __init__(self, side, face, speed, travel, half=(1.6, 1.6, 0.05)):
        self.side, self.face, self.speed, self.travel = float(side), float(face), float(speed), float(travel)
        self.half = np.asarray(half, dtype=np.float32)
        self.idx = np.zeros(0, np.int32)

    def centre(self, t):
        inner = self.face - min(self.speed * t, self.travel)
        return np.array([0.0, 0.0, self.side * (inner + float(self.half[2]))])

    def targets(self, t):
        return np.zeros((0, 3), np.float32)

    def collider(self, t):
        return 1, np.concatenate([np.eye(3).reshape(-1), self.centre(t)]).astype(np.float32), self.half


def dense_contact_scenario(n=4_000_000, seed=0, **kw):
    """The dense-contact stress workload: 12-NN graph, 128-member clusters, two parallel
    plates (box colliders) normal to the thinnest axis (z) closing at 0.005 per frame in
    all (each plate 0.0025) until the gap is 40 % of the initial thickness, then holding;
    self-collision on; 10 substeps x 20 iterations per frame."""
    scene = kw.pop("scene", None) or make_scene(n, seed, knn=12)
    z = scene["pos"][:, 2].astype(np.float64)
    thick = float(z.max() - z.min())
    travel = 0.5 * 0.6 * thick
    plates = [Plate(+1.0, float(z.max()), 0.0025, travel), Plate(-1.0, float(-z.min()), 0.0025, travel)]
    kw.setdefault("self_collision", True)
    kw.setdefault("within_body", True)
    kw.setdefault("iters", 20)
    kw.setdefault("max_members", 128)
    return Scenario(scene, plates, **kw)


class RuntimeScenario:
    """The Isaac runtime's own configuration and call order, on a synthetic object.

    Setup as runtime_loop.py:246-257 (constants at runtime_loop.py:39-71): one solver step
    per 60 Hz frame with dt 1/60 and 16 iterations, distance and volume constraints
    (volume compliance 1e-6, 3-ring candidates, 2048-member cap, leader spacing 2), shape
    matching off with the float polar, object shape keeping 0.9 on the device, ellipsoid
    contacts (``contact_bits``; the runtime's 1 = colliders) with tau 0.2 and a 0.02 cap,
    the ground off and gravity 0 for the first (upload) step, then reset, launch at rest
    and release (runtime_loop.py:402-408).

    Per frame as runtime_loop.py:519-548 and 393-401: the ground plane under the object
    (restitution 0.9, friction 0.5, contact radius 0.003 H and slop 0.002 H of the object
    height H, gravity 5.81) set once, two spherical finger pads as colliders (margin
    0.003 H, friction 0.5), the held Gaussians pinned with the runtime's hold weight, one
    step, the collider statistics, the positions and the deformed shapes (deform eps
    1e-2), which re-pack the contact ellipsoids (xpbd_capi.cu:255-256).

    The pads close on the object along y for ``close`` frames (contact only), then each
    holds the Gaussians within ``hold_radius`` of its centre where they are at that frame
    (``grasp_pos``, read from the solver unless given) and lifts them +z."""

    ITERS, DT, GRAVITY, FRICTION, RESTITUTION, DAMPING = 16, 1.0 / 60.0, 5.81, 0.5, 0.9, 0.01
    CONTACT_TAU, CONTACT_CAP, DEFORM_EPS, HOLD_WEIGHT, OBJECT_SHAPE = 0.2, 0.02, 1e-2, 1.0, 0.9

    def __init__(self, scene, contact_bits=1, close=15, close_speed=0.01, lift_speed=0.004, pad_radius=0.1,
                 pad_gap=0.02, hold_radius=0.13, grasp_pos=None):
        self.scene = scene
        self.contact_bits = int(contact_bits)
        p = scene["pos"].astype(np.float64)
        self.H = float(p[:, 2].max() - p[:, 2].min())
        self.floor = float(p[:, 2].min()) - 0.003 * self.H
        ymax = float(np.abs(p[:, 1]).max())
        self.pad0 = [np.array([0.0, -(ymax + pad_radius + pad_gap), 0.0]),
                     np.array([0.0, ymax + pad_radius + pad_gap, 0.0])]
        self.pad_dir = [np.array([0.0, 1.0, 0.0]), np.array([0.0, -1.0, 0.0])]
        self.close, self.close_speed, self.lift_speed = int(close), float(close_speed), float(lift_speed)
        self.pad_radius, self.hold_radius = float(pad_radius), float(hold_radius)
        self.grasp_pos = grasp_pos
        self.grasp_idx = None
        self.k = 0

    @property
    def n(self):
        return self.scene["pos"].shape[0]

    def pad_centre(self, side, frame):
        t = min(frame, self.close)
        c = self.pad0[side] + self.pad_dir[side] * (self.close_speed * t)
        return c + np.array([0.0, 0.0, self.lift_speed * max(0, frame - self.close)])

    def colliders(self, frame):
        poses = [np.concatenate([np.eye(3).reshape(-1), self.pad_centre(s, frame)]) for s in (0, 1)]
        dims = [[self.pad_radius, 0.0, 0.0]] * 2
        return [0, 0], np.asarray(poses, np.float32), np.asarray(dims, np.float32)

    def setup(self, solver):
        solver.create(self.scene)
        solver.set_solver(iters=self.ITERS, dt=self.DT, under_relax=0.6, vel_damping=self.DAMPING)
        solver.set_constraints(distance=True, shape=False, angle=False, volume=True)
        solver.set_volume(compliance=1e-6, ring_k=3, max_members=2048, leader_min_hop=2)
        solver.set_shape_robust(False)
        solver.set_object_shape(self.OBJECT_SHAPE)
        solver.set_object_shape_gpu(True)
        solver.set_self_collision(False, 1.5, 2.0, False)   # settings outlive create: the runtime's default
        solver.set_colliders([], [], [])   # and so do the colliders' last poses
        solver.volume_stats(False)
        ok = solver.set_contact_shape(self.contact_bits, self.CONTACT_TAU, self.CONTACT_CAP)
        solver.set_ground(False, (0.0, 0.0, 1.0), 0.0, gravity=0.0)
        solver.step()
        solver.reset()
        solver.launch((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 0.0))
        solver.clear_attached()
        self.k = 0
        self.grasp_idx = None
        return ok

    def _hold(self, solver, frame):
        if frame <= self.close:
            return
        if self.grasp_idx is None:
            pos = self.grasp_pos if self.grasp_pos is not None else solver.positions()
            self.grasp_pos = np.asarray(pos, np.float32)
            idx, ref = [], []
            for s in (0, 1):
                c = self.pad_centre(s, self.close)
                d2 = ((self.grasp_pos.astype(np.float64) - c) ** 2).sum(1)
                sel = np.nonzero(d2 <= self.hold_radius ** 2)[0]
                idx.append(sel)
                ref.append(self.grasp_pos[sel].astype(np.float64) - c)
            self.grasp_idx, self.grasp_rel = idx, ref
        idx, pos = [], []
        for s in (0, 1):
            idx.append(self.grasp_idx[s])
            pos.append(self.pad_centre(s, frame) + self.grasp_rel[s])
        idx = np.concatenate(idx).astype(np.int32)
        if len(idx) == 0:
            return
        w = max(1.0, self.HOLD_WEIGHT * (self.n - len(idx)) / len(idx))
        solver.set_attached(idx, np.concatenate(pos).astype(np.float32), w)

    def advance(self, solver, count, record=None):
        """``count`` frames; ``record(solver, frame, shapes)`` after each when given."""
        for _ in range(count):
            if self.k == 0:
                solver.set_ground(True, (0.0, 0.0, 1.0), self.floor, friction=self.FRICTION,
                                  restitution=self.RESTITUTION, contact_radius=0.003 * self.H,
                                  contact_slop=0.002 * self.H, gravity=self.GRAVITY)
            types, poses, dims = self.colliders(self.k + 1)
            solver.set_colliders(types, poses, dims, margin=0.003 * self.H, friction=self.FRICTION)
            self._hold(solver, self.k + 1)
            solver.step()
            self.k += 1
            solver.collider_stats(2)
            shapes = solver.shapes(self.DEFORM_EPS)
            if record is not None:
                record(solver, self.k, shapes)


def bbox_diagonal(pos):
    p = np.asarray(pos, dtype=np.float64)
    return float(np.linalg.norm(p.max(0) - p.min(0)))


# ---------------------------------------------------------------------------
# ChainMail workload (forward.cu:12808-13006): a displacement wave from seeds
# ---------------------------------------------------------------------------
CHAINMAIL_DEFAULTS = dict(prop_iters=20, relax_iters=5, prop_strength=0.5, relax_stiffness=0.99,
                          relax_damping=0.1)   # the reference's tunables (forward.cu:60-64)


def chainmail_scene(n=4000, seed=21):
    """The config-0 ellipsoid with opacity uniform in [0.02, 1): densities fall in all four
    ChainMail classes (air < 0.13 <= skin < 0.45 <= 0.75 <= bone, forward.h:63-65)."""
    sc = make_scene(n, seed)
    sc["opacity"] = np.random.default_rng(seed + 7).uniform(0.02, 1.0, n).astype(np.float32)
    return sc


def chainmail_script(solver, sc, record, push=1.0):
    """Create, one solver step (graph upload), reset to rest; then two waves:
    run 1 — 30 seeds at the -x end pushed +0.02 x, the reference's default sweeps;
    run 2 — 15 seeds at the +x end pushed (-0.015, 0.005, 0), other material constants,
    3 propagation + 2 relax sweeps (the first wave is still travelling).
    ``record(tag)`` is called after each run; ``push`` scales both seed displacements."""
    solver.create(sc)
    solver.step()
    solver.reset()
    pos = sc["pos"].astype(np.float64)
    left = np.argsort(np.linalg.norm(pos - np.array([-0.9, 0.0, 0.0]), axis=1), kind="stable")[:30]
    right = np.argsort(np.linalg.norm(pos - np.array([0.9, 0.0, 0.0]), axis=1), kind="stable")[:15]
    solver.chainmail_set_material()
    solver.chainmail_seed(left, np.tile(np.float32([0.02 * push, 0.0, 0.0]), (len(left), 1)))
    solver.chainmail_run(**CHAINMAIL_DEFAULTS)
    record("run1")
    solver.chainmail_set_material(2.0, 0.2, 0.05, 0.02, True, 0.5)
    solver.chainmail_seed(right, np.tile(np.float32([-0.015 * push, 0.005 * push, 0.0]), (len(right), 1)))
    solver.chainmail_run(3, 2, 0.5, 0.99, 0.1)
    record("run2")
    solver.chainmail_set_material()

