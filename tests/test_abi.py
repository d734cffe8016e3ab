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
    assert L.xpbd_press_start(0, 0.1, 10.0, 1) == -1


def test_graft_entry_has_build_and_smoke():
    import __graft_entry__
    assert callable(__graft_entry__.build) and callable(__graft_entry__.smoke)
