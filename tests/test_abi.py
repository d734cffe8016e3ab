"""The C-ABI libraries load and export every entry point include/xpbd_capi.h declares;
host-side argument checks work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import helpers as H

HEADER = os.path.join(H.ROOT, "include", "xpbd_capi.h")


def declared(prefix=None):
    names = re.findall(r"^XPBD_API[^;(]*?\b(xpbd_\w+)\s*\(", open(HEADER).read(), re.M)
    return [n for n in names if prefix is None or n.startswith(prefix)]


def reference_names():
    return [n for n in declared() if not n.startswith("xpbd_b200_")]


def test_header_declares_reference_abi():
    # the 29 entry points of the reference's C ABI (xpbd_capi.cu:66-310)
    assert len(reference_names()) == 29


def test_product_library_exports_header():
    if not os.path.isfile(H.B200_SO):
        import __graft_entry__
        __graft_entry__.build()
    lib = ctypes.CDLL(H.B200_SO)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_reference_abi():
    lib = ctypes.CDLL(H.ensure_oracle())
    missing = [n for n in reference_names() if not hasattr(lib, n)]
    assert not missing, missing


def test_bridge_binds_product_library():
    x = H.pkg.XPBD()
    assert x.has_attach and x.has_contact_shape


def test_host_side_errors_without_gpu():
    """Calls that fail before touching the device behave like the reference's."""
    x = H.pkg.bridge.XPBD(H.B200_SO)
    L = x.lib
    assert L.xpbd_step() == -1
    assert "xpbd_create first" in x.last_error()
    assert L.xpbd_positions_host(np.zeros(3, np.float32), 1) == -1
    assert "no step yet" in x.last_error()
    assert L.xpbd_set_attached(1, np.zeros(1, np.int32), np.zeros(3, np.float32), 1.0) == -1
    assert L.xpbd_compute_shapes(0.01, np.zeros(3, np.float32), np.zeros(4, np.float32), 1) == -1
    assert L.xpbd_reset() == -1
    assert L.xpbd_positions_device() == 0
    assert L.xpbd_count() == 0
    sc = H.scenes.make_scene(50, 1)
    rc = L.xpbd_create(0, sc["pos"].ravel(), sc["scales"].ravel(), sc["rots"].ravel(), sc["opacity"], 0,
                       np.zeros(2, np.int32), np.zeros(1, np.float32), np.zeros(1, np.float32))
    assert rc == -1 and "invalid arguments" in x.last_error()
    assert L.xpbd_press_start(0, 0.1, 10.0, 1) == -1 and "step once first" in x.last_error()


def test_graft_entry_has_build_and_smoke():
    import __graft_entry__
    assert callable(__graft_entry__.build) and callable(__graft_entry__.smoke)


def reference_checkout():
    """The reference checkout: $XPBD_REFERENCE, else a directory named reference beside
    this repository; None when neither holds src/xpbd_bridge.py."""
    for d in (os.environ.get("XPBD_REFERENCE"), os.path.join(os.path.dirname(H.ROOT), "reference")):
        if d and os.path.isfile(os.path.join(d, "src", "xpbd_bridge.py")):
            return d
    return None


def test_reference_bridge_sets_up_on_product_library():
    """The reference's own, unmodified ctypes bridge (src/xpbd_bridge.py) binds this
    library and runs the runtime's setup calls up to the first step (runtime_loop.py:
    246-257): create, solver, constraint, volume, shape and object settings, and the
    ellipsoid contact shapes, which report True (runtime_loop.py:253 falls back to point
    contact on False and raises on an error)."""
    import importlib
    import sys
    ref = reference_checkout()
    if ref is None:
        pytest.skip("no reference checkout (set XPBD_REFERENCE)")
    sys.path.insert(0, os.path.join(ref, "src"))
    try:
        xb = importlib.import_module("xpbd_bridge")
    finally:
        sys.path.pop(0)
    sim = xb.XPBD(H.B200_SO)
    assert sim.has_attach and sim.has_contact_shape
    sc = H.scenes.make_scene(400, 3)
    sim.create(sc)
    assert sim.lib.xpbd_count() == 400
    sim.set_solver(iters=16, dt=1 / 60, under_relax=0.6, vel_damping=0.01)
    sim.set_constraints(distance=True, shape=False, angle=False, volume=True)
    sim.set_volume(compliance=1e-6, ring_k=3, max_members=2048, leader_min_hop=2)
    sim.set_shape_robust(False)
    sim.set_object_shape(0.9)
    sim.set_object_shape_gpu(True)
    assert sim.set_contact_shape(1, 0.2, 0.02) is True
    sim.set_ground(False, (0.0, 0.0, 1.0), 0.0, gravity=0.0)
    sim.destroy()
    with pytest.raises(RuntimeError, match="create first"):
        sim.set_contact_shape(1, 0.2, 0.02)
