"""The allocation-free self-collision build (xpbd_b200_selfcol_candidates_static).

Some callers of this library cannot allocate device memory: a host application that
owns the whole device heap hands its plug-ins buffers and forbids cudaMalloc, whose
implicit device synchronisation would stall its frame.  For them the library offers
the once-per-step self-collision candidate build on caller-owned device buffers, with
all scratch in a static device array (up to 65,536 particles).  This test checks,
through the C ABI, that two calls in a row give the same candidate counts and lists as
the solver's own allocating build (xpbd_b200_selfcol_build) on the same positions, and
that sizes beyond the limit are refused.  (The test itself allocates its input and
output buffers with torch; only the entry point must not allocate.)

It is collected last (file name) so that a run stopping at the first failure has run
every other test first; it passes alone and after the other tests.
"""
import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _static_fn(lib):
    f = lib.xpbd_b200_selfcol_candidates_static
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                  ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_static_scratch_build_matches_allocating_build():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    lib = H.b200()
    static_build = _static_fn(lib.lib)
    sc, grippers = H.two_blob_scene()
    s = H.scenes.Scenario(sc, grippers, self_collision=True, within_body=True)
    s.setup(lib)
    s.advance(lib, 3)
    n = s.n
    spacing = float(lib.floats("self_col")[0])
    obj = lib.ints("obj_id")
    rest4 = np.zeros((n, 4), np.float32)
    rest4[:, :3] = sc["pos"]
    dev = torch.device("cuda:0")
    d_rest = torch.from_numpy(rest4).to(dev)
    d_obj = torch.from_numpy(obj.astype(np.int32)).to(dev)
    d_contacts = torch.full((n * 32,), -7, dtype=torch.int32, device=dev)
    d_counts = torch.full((n,), -7, dtype=torch.int32, device=dev)
    d_total = torch.zeros(1, dtype=torch.int32, device=dev)
    rng = np.random.default_rng(5)
    x0 = lib.positions()
    # two calls in a row on different states; the second sees what the first left
    for call in range(2):
        x = (x0 + rng.normal(0.0, 0.002, x0.shape)).astype(np.float32)
        # bodies pushed together: the predicted state overlaps across the gap
        p = x.copy()
        p[:, 0] -= np.sign(p[:, 0]) * np.float32(0.05 + 0.02 * call)
        expected_total = lib.selfcol_build(x, p)
        exp_counts = lib.ints("sc_count")
        exp_contacts = lib.ints("sc_contact")
        assert expected_total > 0
        x4 = np.zeros((n, 4), np.float32)
        p4 = np.zeros((n, 4), np.float32)
        x4[:, :3] = x
        p4[:, :3] = p
        d_x = torch.from_numpy(x4).to(dev)
        d_p = torch.from_numpy(p4).to(dev)
        stream = torch.cuda.current_stream(dev)
        rc = static_build(n, d_x.data_ptr(), d_p.data_ptr(), d_rest.data_ptr(), d_obj.data_ptr(), spacing, 1.5, 2.0, 1,
                          d_contacts.data_ptr(), d_counts.data_ptr(), d_total.data_ptr(), stream.cuda_stream)
        assert rc == 0, lib.last_error()
        torch.cuda.synchronize()
        counts = d_counts.cpu().numpy()
        contacts = d_contacts.cpu().numpy()
        assert int(d_total.cpu().item()) == expected_total
        assert H.contacts_equal(counts, contacts, exp_counts, exp_contacts), f"call {call}"
    lib.destroy()


def test_static_scratch_build_one_object_without_ids():
    """obj_id = NULL (one object: the ids are zeroed in the scratch array) against the
    allocating build of a single-object scene, two calls in a row."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required")
    lib = H.b200()
    static_build = _static_fn(lib.lib)
    s = H.scenes.plain_scene_scenario(6000, 4, pins=30, self_collision=True, within_body=True)
    s.setup(lib)
    s.advance(lib, 2)
    n = s.n
    spacing = float(lib.floats("self_col")[0])
    dev = torch.device("cuda:0")
    rest4 = np.zeros((n, 4), np.float32)
    rest4[:, :3] = s.scene["pos"]
    d_rest = torch.from_numpy(rest4).to(dev)
    d_contacts = torch.full((n * 32,), -7, dtype=torch.int32, device=dev)
    d_counts = torch.full((n,), -7, dtype=torch.int32, device=dev)
    d_total = torch.zeros(1, dtype=torch.int32, device=dev)
    x0 = lib.positions()
    rng = np.random.default_rng(9)
    for call in range(2):
        x = (x0 + rng.normal(0.0, 0.003, x0.shape)).astype(np.float32)
        p = (x + rng.normal(0.0, 0.004 * (call + 1), x.shape)).astype(np.float32)
        expected_total = lib.selfcol_build(x, p)
        exp_counts, exp_contacts = lib.ints("sc_count"), lib.ints("sc_contact")
        assert expected_total > 0
        x4 = np.zeros((n, 4), np.float32)
        p4 = np.zeros((n, 4), np.float32)
        x4[:, :3], p4[:, :3] = x, p
        d_x, d_p = torch.from_numpy(x4).to(dev), torch.from_numpy(p4).to(dev)
        rc = static_build(n, d_x.data_ptr(), d_p.data_ptr(), d_rest.data_ptr(), None, spacing, 1.5, 2.0, 1,
                          d_contacts.data_ptr(), d_counts.data_ptr(), d_total.data_ptr(),
                          torch.cuda.current_stream(dev).cuda_stream)
        assert rc == 0, lib.last_error()
        torch.cuda.synchronize()
        assert int(d_total.cpu().item()) == expected_total
        assert H.contacts_equal(d_counts.cpu().numpy(), d_contacts.cpu().numpy(), exp_counts, exp_contacts), call
    lib.destroy()


def test_static_scratch_limit_is_enforced():
    lib = H.b200()
    static_build = _static_fn(lib.lib)
    rc = static_build(65537, 1, 1, 1, None, 0.01, 1.5, 2.0, 1, 1, 1, None, None)
    assert rc == -1 and "65536" in lib.last_error()
    rc = static_build(100, 1, 1, 1, None, 0.0, 1.5, 2.0, 1, 1, 1, None, None)
    assert rc == -1 and "spacing" in lib.last_error()
