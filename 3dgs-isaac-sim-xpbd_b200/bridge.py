"""ctypes binding of the ``xpbd_*`` C ABI.

The class mirrors the caller side of the reference (src/xpbd_bridge.py:45-271):
the same method names, argument meanings, defaults and error behaviour (an ``int``
status of ``-1`` raises ``RuntimeError`` carrying ``xpbd_last_error()``).  It binds
any shared library that exports the ABI declared in ``include/xpbd_capi.h`` — this
package's CUDA library, and, in the test-suite, the parity oracles.

Positions, scales and quaternions are in the caller's Gaussian order (PLY/USD order,
xpbd_capi.cu:4-5).
"""
import ctypes
import os

import numpy as np

_F32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_I32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def bind_abi(lib):
    """Declare argtypes/restypes of the 29 reference entry points on ``lib``
    (signatures as xpbd_capi.cu:66-310 and xpbd_bridge.py:58-112)."""
    c_int, c_float = ctypes.c_int, ctypes.c_float
    L = lib
    L.xpbd_last_error.restype = ctypes.c_char_p
    L.xpbd_create.argtypes = [c_int, _F32, _F32, _F32, _F32, c_int, _I32, _F32, _F32]
    L.xpbd_create.restype = c_int
    L.xpbd_destroy.restype = None
    L.xpbd_count.restype = c_int
    L.xpbd_set_solver.argtypes = [c_int] + [c_float] * 10
    L.xpbd_set_solver.restype = None
    L.xpbd_set_constraints.argtypes = [c_int] * 4
    L.xpbd_set_constraints.restype = None
    L.xpbd_set_volume.argtypes = [c_float, c_int, c_int, c_int]
    L.xpbd_set_volume.restype = None
    L.xpbd_set_ground.argtypes = [c_int] + [c_float] * 9
    L.xpbd_set_ground.restype = None
    L.xpbd_set_object_shape.argtypes = [c_float]
    L.xpbd_set_object_shape.restype = None
    L.xpbd_set_shape_robust.argtypes = [c_int]
    L.xpbd_set_shape_robust.restype = None
    L.xpbd_set_object_shape_gpu.argtypes = [c_int]
    L.xpbd_set_object_shape_gpu.restype = None
    L.xpbd_set_self_collision.argtypes = [c_int, c_float, c_float, c_int]
    L.xpbd_set_self_collision.restype = None
    L.xpbd_self_collision_stats.argtypes = [_I32]
    L.xpbd_self_collision_stats.restype = None
    L.xpbd_set_colliders.argtypes = [c_int, _I32, _F32, _F32, c_float, c_float]
    L.xpbd_set_colliders.restype = None
    L.xpbd_collider_stats.argtypes = [_I32, _F32, _F32, c_int]
    L.xpbd_collider_stats.restype = c_int
    L.xpbd_add_rigid_velocity.argtypes = [_F32, _F32, _F32]
    L.xpbd_add_rigid_velocity.restype = c_int
    L.xpbd_set_attached.argtypes = [c_int, _I32, _F32, c_float]
    L.xpbd_set_attached.restype = c_int
    L.xpbd_set_contact_shape.argtypes = [c_int, c_float, c_float]
    L.xpbd_set_contact_shape.restype = c_int
    L.xpbd_step.restype = c_int
    L.xpbd_positions_device.restype = ctypes.c_ulonglong
    L.xpbd_positions_host.argtypes = [_F32, c_int]
    L.xpbd_positions_host.restype = c_int
    L.xpbd_reset.restype = c_int
    L.xpbd_launch.argtypes = [_F32, _F32, _F32]
    L.xpbd_launch.restype = c_int
    L.xpbd_volume_stats.argtypes = [c_int, ctypes.POINTER(c_float), ctypes.POINTER(c_float)]
    L.xpbd_volume_stats.restype = None
    L.xpbd_compute_shapes.argtypes = [c_float, _F32, _F32, c_int]
    L.xpbd_compute_shapes.restype = c_int
    L.xpbd_press_start.argtypes = [c_int, c_float, c_float, c_int]
    L.xpbd_press_start.restype = c_int
    L.xpbd_press_stop.restype = None
    L.xpbd_press_autolog.argtypes = [c_int]
    L.xpbd_press_autolog.restype = None
    L.xpbd_press_state.argtypes = [ctypes.POINTER(c_float)] * 4
    L.xpbd_press_state.restype = c_int
    return L


class _Selected:
    """Forwards ABI calls to a library after selecting one engine handle for the thread."""

    def __init__(self, lib, handle):
        self._lib = lib
        self._handle = handle

    def __getattr__(self, name):
        f = getattr(self._lib, name)
        if not callable(f) or name.startswith("xpbd_b200_engine_"):
            return f
        lib, handle = self._lib, self._handle

        def call(*args):
            lib.xpbd_b200_engine_select(handle)
            return f(*args)
        return call


_LIBS = {}


def load(dll_path):
    """One ctypes handle per library path (every XPBD object shares it)."""
    path = os.path.abspath(dll_path)
    if path not in _LIBS:
        if not os.path.isfile(path):
            raise FileNotFoundError(f"XPBD library not found: {path}")
        _LIBS[path] = bind_abi(ctypes.CDLL(path))
    return _LIBS[path]


class XPBD:
    """One solver instance behind the ``xpbd_*`` ABI of ``dll_path``: the library's
    singleton, or — with ``instance=True`` on a library exporting the engine-handle
    extension — a separate resident engine of its own."""

    SPHERE, BOX, CAPSULE = 0, 1, 2

    def __init__(self, dll_path, instance=False):
        lib = load(dll_path)
        self.handle = None
        if instance:
            lib.xpbd_b200_engine_new.restype = ctypes.c_void_p
            lib.xpbd_b200_engine_free.argtypes = [ctypes.c_void_p]
            lib.xpbd_b200_engine_select.argtypes = [ctypes.c_void_p]
            self.handle = lib.xpbd_b200_engine_new()
            if not self.handle:
                raise MemoryError("xpbd_b200_engine_new failed")
            self.lib = _Selected(lib, self.handle)
        else:
            self.lib = lib
        self.raw = lib
        self.path = dll_path
        self.has_attach = hasattr(self.lib, "xpbd_set_attached")
        self.has_contact_shape = hasattr(self.lib, "xpbd_set_contact_shape")
        self.n = 0

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {self.last_error()}")

    def last_error(self):
        return self.lib.xpbd_last_error().decode(errors="replace")

    def create(self, inp):
        e = inp["edges"].shape[0]
        edges = np.ascontiguousarray(inp["edges"], dtype=np.int32).ravel()
        if e == 0:
            edges = np.zeros(2, np.int32)
        self._check(self.lib.xpbd_create(
            inp["pos"].shape[0],
            np.ascontiguousarray(inp["pos"], dtype=np.float32).ravel(),
            np.ascontiguousarray(inp["scales"], dtype=np.float32).ravel(),
            np.ascontiguousarray(inp["rots"], dtype=np.float32).ravel(),
            np.ascontiguousarray(inp["opacity"], dtype=np.float32),
            e, edges,
            np.ascontiguousarray(inp["rest"], dtype=np.float32) if e else np.zeros(1, np.float32),
            np.ascontiguousarray(inp["stiff"], dtype=np.float32) if e else np.zeros(1, np.float32)),
            "xpbd_create")
        self.n = inp["pos"].shape[0]

    def set_solver(self, iters=20, dt=1 / 60, under_relax=0.6, vel_damping=0.01, stiffness_scale=1.0,
                   inv_mass_scale=1.0, dist_compliance=0.0, shape_compliance=0.0, shape_blend=0.1,
                   angle_compliance=1e-2, angle_blend=0.2):
        self.lib.xpbd_set_solver(int(iters), dt, under_relax, vel_damping, stiffness_scale, inv_mass_scale,
                                 dist_compliance, shape_compliance, shape_blend, angle_compliance, angle_blend)

    def set_constraints(self, distance=True, shape=True, angle=False, volume=True):
        self.lib.xpbd_set_constraints(int(distance), int(shape), int(angle), int(volume))

    def set_volume(self, compliance=1e-6, ring_k=3, max_members=2048, leader_min_hop=2):
        self.lib.xpbd_set_volume(compliance, int(ring_k), int(max_members), int(leader_min_hop))

    def set_ground(self, enabled, up, height, friction=0.5, restitution=0.0, contact_radius=0.0,
                   contact_slop=0.0, gravity=0.0):
        self.lib.xpbd_set_ground(int(enabled), float(up[0]), float(up[1]), float(up[2]), height, friction,
                                 restitution, contact_radius, contact_slop, gravity)

    def set_object_shape(self, stiffness):
        self.lib.xpbd_set_object_shape(stiffness)

    def set_object_shape_gpu(self, enabled):
        self.lib.xpbd_set_object_shape_gpu(int(enabled))

    def set_colliders(self, types, poses, dims, margin=0.0, friction=0.0):
        """Kinematic colliders (K,) types 0 sphere / 1 box / 2 capsule; poses (K,12) local->world
        rotation row-major + centre; dims (K,3).  An empty list disables all colliders."""
        types = np.ascontiguousarray(np.asarray(types, dtype=np.int32).reshape(-1))
        k = len(types)
        poses = np.ascontiguousarray(np.asarray(poses, dtype=np.float32).reshape(k, 12)
                                     if k else np.zeros((1, 12), np.float32))
        dims = np.ascontiguousarray(np.asarray(dims, dtype=np.float32).reshape(k, 3)
                                    if k else np.zeros((1, 3), np.float32))
        if not k:
            types = np.zeros(1, dtype=np.int32)
        self.lib.xpbd_set_colliders(k, types, poses.ravel(), dims.ravel(), float(margin), float(friction))

    def collider_stats(self, count):
        hits = np.zeros(max(count, 1), dtype=np.int32)
        push = np.zeros(max(count, 1) * 3, dtype=np.float32)
        cen = np.zeros(max(count, 1) * 3, dtype=np.float32)
        n = self.lib.xpbd_collider_stats(hits, push, cen, count)
        return hits[:n], push[:3 * n].reshape(n, 3), cen[:3 * n].reshape(n, 3)

    def add_rigid_velocity(self, dv, dw=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (dv, dw, center)]
        self._check(self.lib.xpbd_add_rigid_velocity(*a), "xpbd_add_rigid_velocity")

    def set_attached(self, idx, pos, weight=1.0):
        idx = np.ascontiguousarray(idx, dtype=np.int32).ravel()
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        self._check(self.lib.xpbd_set_attached(len(idx), idx, pos.ravel(), float(weight)), "xpbd_set_attached")

    def clear_attached(self):
        self._check(self.lib.xpbd_set_attached(0, np.zeros(1, np.int32), np.zeros(3, np.float32), 1.0),
                    "xpbd_set_attached")

    def set_contact_shape(self, enabled, tau=0.2, radius_cap=0.0):
        self._check(self.lib.xpbd_set_contact_shape(int(enabled), float(tau), float(radius_cap)),
                    "xpbd_set_contact_shape")
        return True

    def set_self_collision(self, enabled, radius_scale=1.5, exclude_scale=2.0, within_body=False):
        self.lib.xpbd_set_self_collision(int(enabled), radius_scale, exclude_scale, int(within_body))

    def self_collision_stats(self):
        """(candidates, active particles, over-cap replacements) of the last step."""
        out = np.zeros(3, dtype=np.int32)
        self.lib.xpbd_self_collision_stats(out)
        return int(out[0]), int(out[1]), int(out[2])

    def set_shape_robust(self, enabled):
        self.lib.xpbd_set_shape_robust(int(enabled))

    def step(self):
        self._check(self.lib.xpbd_step(), "xpbd_step")

    def positions(self):
        out = np.empty((self.n, 3), dtype=np.float32)
        self._check(self.lib.xpbd_positions_host(out.ravel(), self.n), "xpbd_positions_host")
        return out

    def shapes(self, deform_eps=1e-2):
        sc = np.empty((self.n, 3), dtype=np.float32)
        q = np.empty((self.n, 4), dtype=np.float32)
        k = self.lib.xpbd_compute_shapes(float(deform_eps), sc.ravel(), q.ravel(), self.n)
        if k < 0:
            self._check(-1, "xpbd_compute_shapes")
        return sc, q, k

    def positions_device_ptr(self):
        return int(self.lib.xpbd_positions_device())

    def reset(self):
        self._check(self.lib.xpbd_reset(), "xpbd_reset")

    def launch(self, lin=(0, 0, 0), ang=(0, 0, 0), tilt=(0, 0, 0)):
        a = [np.ascontiguousarray(v, dtype=np.float32) for v in (lin, ang, tilt)]
        self._check(self.lib.xpbd_launch(*a), "xpbd_launch")

    def volume_stats(self, enable=True):
        m, s = ctypes.c_float(0.0), ctypes.c_float(0.0)
        self.lib.xpbd_volume_stats(int(enable), ctypes.byref(m), ctypes.byref(s))
        return m.value, s.value

    # ---- ChainMail (forward.cu:12808-13006; not in the reference C ABI) ----
    # entry points xpbd_b200_chainmail_*; a subclass binding another library with the
    # same signatures under another prefix sets CHAINMAIL_PREFIX
    CHAINMAIL_PREFIX = "xpbd_b200_"

    def _cm(self, name, argtypes, restype):
        prefix = self.CHAINMAIL_PREFIX
        f = getattr(self.raw, prefix + name, None)
        if f is None:
            raise AttributeError(f"{self.path} has no ChainMail entry point {prefix}{name}")
        f.argtypes = argtypes       # on the ctypes function; self.lib may be an engine proxy
        f.restype = restype
        return prefix, getattr(self.lib, prefix + name)

    def chainmail_set_material(self, global_scale=1.0, air=0.1, skin=0.1, bone=0.1, use_edge_stiffness=True,
                               edge_influence=1.0):
        _, f = self._cm("chainmail_set_material", [ctypes.c_float] * 4 + [ctypes.c_int, ctypes.c_float], None)
        f(global_scale, air, skin, bone, int(use_edge_stiffness), edge_influence)

    def chainmail_seed(self, idx, delta):
        """Seeds start the wave: each moves by its delta (K, 3) and gets arrival time 0."""
        idx = np.ascontiguousarray(idx, dtype=np.int32).reshape(-1)
        delta = np.ascontiguousarray(delta, dtype=np.float32).reshape(-1, 3)
        _, f = self._cm("chainmail_seed", [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int)
        self._check(f(len(idx), idx.ctypes.data, delta.ctypes.data), "chainmail_seed")

    def chainmail_run(self, prop_iters=20, relax_iters=5, prop_strength=0.5, relax_stiffness=0.99, relax_damping=0.1):
        """Propagation and relax sweeps; defaults are the reference's (forward.cu:60-64)."""
        _, f = self._cm("chainmail_run", [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 3, ctypes.c_int)
        self._check(f(prop_iters, relax_iters, prop_strength, relax_stiffness, relax_damping), "chainmail_run")

    def chainmail_times(self):
        """Arrival times (N,), 1e9 where the wave has not arrived."""
        out = np.zeros(max(self.n, 1), np.float32)
        _, f = self._cm("chainmail_times", [ctypes.c_void_p, ctypes.c_int], ctypes.c_int)
        got = f(out.ctypes.data, out.size)
        if got != self.n:
            raise RuntimeError(f"chainmail_times: {self.last_error()}")
        return out[:self.n]

    # ---- splatting into a device image (the viewer's rasteriser; library only) ----
    def _ext(self, name, argtypes, restype):
        f = getattr(self.raw, "xpbd_b200_" + name, None)
        if f is None:
            raise AttributeError(f"{self.path} has no entry point xpbd_b200_{name}")
        f.argtypes = argtypes
        f.restype = restype
        return getattr(self.lib, "xpbd_b200_" + name)

    def render_set_colors(self, colors, sh_degree=-1):
        """RGB (N, 3) with sh_degree -1, else SH coefficients (N, (d+1)^2, 3)."""
        c = np.ascontiguousarray(colors, dtype=np.float32)
        f = self._ext("render_set_colors", [ctypes.c_int, ctypes.c_int, ctypes.c_void_p], ctypes.c_int)
        self._check(f(self.n, int(sh_degree), c.ctypes.data), "render_set_colors")
        self._keep_colors = c

    def render_set_options(self, antialiasing=False, box=None, pick=False):
        f = self._ext("render_set_options", [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int], None)
        if box is None:
            f(int(antialiasing), None, None, int(pick))
        else:
            lo = np.ascontiguousarray(box[0], dtype=np.float32)
            hi = np.ascontiguousarray(box[1], dtype=np.float32)
            f(int(antialiasing), lo.ctypes.data, hi.ctypes.data, int(pick))

    def render_set_floor(self, visible, origin=(0.0, 0.0, 0.0), checker=1.0, fade_radius=10.0):
        o = np.ascontiguousarray(origin, dtype=np.float32)
        f = self._ext("render_set_floor", [ctypes.c_int, ctypes.c_void_p, ctypes.c_float, ctypes.c_float], None)
        f(int(visible), o.ctypes.data, float(checker), float(fade_radius))

    def render(self, cam, deform_eps=1e-2, bg=(0.0, 0.0, 0.0), scale_modifier=1.0, to_host=True):
        """One frame of the current state through ``cam`` (splat.Camera).  Returns
        (image (3, H, W) float32 or None, number of (tile, Gaussian) pairs)."""
        f = self._ext("render", [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 4
                      + [ctypes.c_void_p, ctypes.c_void_p], ctypes.c_longlong)
        bgv = np.ascontiguousarray(bg, dtype=np.float32)
        out = np.empty((3, cam.height, cam.width), np.float32) if to_host else None
        m = f(cam.view.ctypes.data, cam.proj.ctypes.data, cam.campos.ctypes.data, cam.width, cam.height,
              cam.tan_fovx, cam.tan_fovy, float(scale_modifier), float(deform_eps), bgv.ctypes.data,
              out.ctypes.data if to_host else None)
        if m < 0:
            self._check(-1, "render")
        return out, int(m)

    def render_device_ptr(self):
        return int(self._ext("render_device", [], ctypes.c_ulonglong)())

    def render_aux(self, width, height, pick=False):
        """final_T (H, W), n_contrib (H, W), picked ids (H, W) or None, radii (N,)."""
        f = self._ext("render_aux", [ctypes.c_void_p] * 3 + [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_int],
                      ctypes.c_int)
        ft = np.empty((height, width), np.float32)
        nc = np.empty((height, width), np.int32)
        pk = np.empty((height, width), np.int32) if pick else None
        radii = np.empty(self.n, np.int32)
        self._check(f(ft.ctypes.data, nc.ctypes.data, pk.ctypes.data if pick else None, width * height,
                      radii.ctypes.data, self.n), "render_aux")
        return ft, nc, pk, radii

    def press_start(self, axis, ramp_per_sec, max_disp_pct, from_lo):
        self._check(self.lib.xpbd_press_start(int(axis), float(ramp_per_sec), float(max_disp_pct), int(from_lo)),
                    "xpbd_press_start")

    def press_autolog(self, enabled):
        self.lib.xpbd_press_autolog(int(enabled))

    def press_stop(self):
        self.lib.xpbd_press_stop()

    def press_state(self):
        v = [ctypes.c_float(0.0) for _ in range(4)]
        active = self.lib.xpbd_press_state(*[ctypes.byref(x) for x in v])
        return bool(active), v[0].value, v[1].value, v[2].value, v[3].value

    def destroy(self):
        self.lib.xpbd_destroy()
        self.n = 0

    def close(self):
        """Release a separate engine (instance=True); the singleton stays."""
        self.destroy()
        if self.handle:
            self.raw.xpbd_b200_engine_free(self.handle)
            self.handle = None


class Arena:
    """A serving arena (xpbd_b200_arena_*): many sessions resident in one engine's buffers
    and advanced together, one launch sequence per substep.  Capacities are in rows
    (Gaussians), directed graph edges, cluster members and reverse-list entries.  A
    session joins with ``admit(solver)`` — an ``XPBD(instance=True)`` engine that has built
    its scene and taken its first step — and leaves with ``retire(slot)``; all sessions
    must share the solver settings."""

    def __init__(self, dll_path, rows, edges, members, rev):
        L = load(dll_path)
        L.xpbd_b200_arena_new.argtypes = [ctypes.c_longlong] * 4
        L.xpbd_b200_arena_new.restype = ctypes.c_void_p
        L.xpbd_b200_arena_admit.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.xpbd_b200_arena_retire.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.xpbd_b200_arena_step.argtypes = ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4
                                           + [ctypes.c_float] * 2 + [ctypes.c_int] + [ctypes.c_void_p] * 3)
        L.xpbd_b200_arena_positions.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.xpbd_b200_arena_sync.argtypes = [ctypes.c_void_p]
        L.xpbd_b200_arena_usage.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.xpbd_b200_arena_free.argtypes = [ctypes.c_void_p]
        L.xpbd_b200_arena_free.restype = None
        self.lib = L
        self.handle = L.xpbd_b200_arena_new(int(rows), int(edges), int(members), int(rev))
        if not self.handle:
            raise RuntimeError(f"xpbd_b200_arena_new: {L.xpbd_last_error().decode(errors='replace')}")

    def _err(self, what):
        return RuntimeError(f"{what}: {self.lib.xpbd_last_error().decode(errors='replace')}")

    def admit(self, solver):
        """The session's slot, or None when it does not fit (retire sessions first)."""
        slot = self.lib.xpbd_b200_arena_admit(self.handle, solver.handle)
        if slot == -2:
            return None
        if slot < 0:
            raise self._err("xpbd_b200_arena_admit")
        return slot

    def retire(self, slot):
        if self.lib.xpbd_b200_arena_retire(self.handle, int(slot)) != 0:
            raise self._err("xpbd_b200_arena_retire")

    def step(self, k, types, poses, dims, col_slot, pin_slot, pin_idx, targets, margin=0.0, friction=0.0):
        """Enqueue k substeps of every live session: colliders ``types`` (C,), ``poses``
        (k, C, 12), ``dims`` (C, 3) acting on the sessions ``col_slot`` (C,); pins of
        session ``pin_slot`` (P,), Gaussian ``pin_idx`` (P,, the session's own order) at
        ``targets`` (k, P, 3)."""
        a = [np.ascontiguousarray(types, np.int32), np.ascontiguousarray(poses, np.float32),
             np.ascontiguousarray(dims, np.float32), np.ascontiguousarray(col_slot, np.int32),
             np.ascontiguousarray(pin_slot, np.int32), np.ascontiguousarray(pin_idx, np.int32),
             np.ascontiguousarray(targets, np.float32)]
        rc = self.lib.xpbd_b200_arena_step(self.handle, int(k), len(a[0]), a[0].ctypes.data, a[1].ctypes.data,
                                           a[2].ctypes.data, a[3].ctypes.data, float(margin), float(friction),
                                           len(a[4]), a[4].ctypes.data, a[5].ctypes.data, a[6].ctypes.data)
        if rc != 0:
            raise self._err("xpbd_b200_arena_step")

    def positions(self, slot, n):
        out = np.empty((n, 3), np.float32)
        if self.lib.xpbd_b200_arena_positions(self.handle, int(slot), out.ctypes.data, int(n)) != 0:
            raise self._err("xpbd_b200_arena_positions")
        return out

    def sync(self):
        if self.lib.xpbd_b200_arena_sync(self.handle) != 0:
            raise self._err("xpbd_b200_arena_sync")

    def usage(self):
        """rows used / capacity, edges, members, reverse entries, live Gaussians, sessions."""
        out = np.zeros(10, np.int64)
        self.lib.xpbd_b200_arena_usage(self.handle, out.ctypes.data)
        keys = ("rows", "rows_cap", "edges", "edges_cap", "members", "members_cap", "rev", "rev_cap", "live", "sessions")
        return dict(zip(keys, (int(v) for v in out)))

    def close(self):
        if self.handle:
            self.lib.xpbd_b200_arena_free(self.handle)
            self.handle = None
