"""The CPU oracle pinned against golden vectors produced by the reference solver itself.

Integer artefacts (graph CSR, cluster membership, transposed membership, both
colourings, self-collision hash keys / sorted order / cell ranges / candidate lists)
must be bit-exact; FP32 positions within 1e-5 of the bounding-box diagonal after one
step and 1e-4 after 100; deformed-shape covariances within 1e-3 relative (p99).
"""
import numpy as np
import pytest

import helpers as H

GRAPH_INT = ["nbr_offset", "nbr_count", "nbr_idx", "vol_offset", "vol_count", "vol_idx", "rev_offset", "rev_count",
             "rev_idx", "mat_type", "gs_edge", "gs_color_offset", "vol_gs_order", "vol_gs_color_offset"]
GRAPH_FLOAT = ["det_rest", "sigma_rest", "v_rest", "rest_len", "gs_rest", "gs_stiff"]


@pytest.fixture(scope="module")
def orc():
    o = H.oracle()
    yield o
    o.destroy()


@pytest.mark.parametrize("case", ["graph_n3000_r1", "graph_n3000_r2", "graph_n3000_k1"])
def test_cluster_topology_bit_exact(orc, case):
    g = H.load_golden(case)
    sc = H.golden_scene(g)
    s = H.scenes.Scenario(sc, [], ring_k=int(g["ring_k"]), max_members=int(g["cap"]),
                          leader_min_hop=int(g["leader"]))
    s.setup(orc)
    orc.step()
    for name in GRAPH_INT:
        np.testing.assert_array_equal(orc.ints(name), g[name], err_msg=name)
    for name in GRAPH_FLOAT:
        a, b = orc.floats(name), g[name]
        assert a.shape == b.shape, name
        np.testing.assert_allclose(a, b, rtol=2e-5, atol=1e-6 * float(np.abs(b).max()), err_msg=name)
    assert H.max_err_over_diag(orc.positions(), g["pos_step1"], H.scenes.bbox_diagonal(sc["pos"])) < H.TOL_1STEP


@pytest.mark.parametrize("case", ["plain_n4000", "plain_n4000_k1", "plain_n4000_fpolar", "plain_n4000_gs",
                                  "object_plain_n4000"])
def test_scenario_positions(orc, case):
    g = H.load_golden(case)
    s = H.scenario_for(case)
    np.testing.assert_array_equal(s.scene["pos"], g["in_pos"])
    np.testing.assert_array_equal(s.scene["edges"], g["in_edges"])
    s.setup(orc)
    orc.set_gs(*((1, 1) if case.endswith("_gs") else (0, 0)))
    orc.volume_stats(True)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    done = 0
    for c in g["checkpoints"]:
        s.advance(orc, int(c) - done)
        done = int(c)
        tol = H.TOL_1STEP if c == 1 else H.TOL_100STEP
        assert H.max_err_over_diag(orc.positions(), g[f"pos_{c}"], diag) < tol, c
        np.testing.assert_allclose(orc.volume_stats(True), g[f"jvw_{c}"], rtol=1e-4, atol=1e-6)
        hits, _, _ = orc.collider_stats(2)
        np.testing.assert_array_equal(hits, g[f"col_hits_{c}"])
    sc_, q_, k_ = orc.shapes(float(g["deform_eps"]))
    assert k_ == int(g["shape_deformed"])
    rel = H.covariance_rel_err(sc_, q_, g["shape_scales"], g["shape_quats"])
    assert np.percentile(rel, 99) < 1e-3 and rel.max() < 1e-2
    orc.set_gs(0, 0)


def test_plain_small_scene_100_frames_first_checkpoints(orc):
    """The 20,000-Gaussian plain workload: first step and first 10 frames."""
    g = H.load_golden("plain_n20000")
    s = H.scenario_for("plain_n20000")
    s.setup(orc)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    s.advance(orc, 1)
    assert H.max_err_over_diag(orc.positions(), g["pos_1"], diag) < H.TOL_1STEP
    s.advance(orc, 99)
    assert H.max_err_over_diag(orc.positions(), g["pos_100"], diag) < H.TOL_100STEP


def test_self_collision_stage_bit_exact(orc):
    g = H.load_golden("selfcol_blobs")
    s = H.scenario_for("selfcol_blobs")
    np.testing.assert_array_equal(s.scene["pos"], g["in_pos"])
    s.setup(orc)
    s.advance(orc, 1)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    assert H.max_err_over_diag(orc.positions(), g["pos_1"], diag) < H.TOL_1STEP
    s.advance(orc, 49)
    # contact dynamics amplify rounding once bodies touch; 50 substeps is before that
    assert H.max_err_over_diag(orc.positions(), g["pos_50"], diag) < H.TOL_100STEP
    assert orc.self_collision_stats()[0] == int(g["sc_stats_50"][0])
    total = orc.selfcol_build(g["stage_x"], g["stage_p"])
    assert total == int(g["stage_total"])
    np.testing.assert_array_equal(orc.floats("self_col"), g["self_col_params"])
    for name in ["sc_keys", "sc_keys_sorted", "sc_idx_sorted", "sc_count", "obj_id"]:
        np.testing.assert_array_equal(orc.ints(name), g[name], err_msg=name)
    assert H.cells_equal(orc.ints("sc_cell_start"), orc.ints("sc_cell_end"), g["sc_cell_start"], g["sc_cell_end"])
    assert H.contacts_equal(orc.ints("sc_count"), orc.ints("sc_contact"), g["sc_count"], g["sc_contact"])


def test_ground_launch_reset(orc):
    g = H.load_golden("misc_n2000")
    sc = H.golden_scene(g)
    s = H.scenes.Scenario(sc, [])
    orc.set_colliders([], [], [])
    s.setup(orc)
    diag = H.scenes.bbox_diagonal(sc["pos"])
    orc.step()
    orc.set_ground(True, (0.0, 0.0, 1.0), -0.45, 0.5, 0.3, 0.0, 0.0, 9.8)
    orc.launch((0.0, 0.0, -1.0), (0.0, 0.0, 2.0), (0.3, 0.0, 0.0))
    assert H.max_err_over_diag(orc.positions(), g["pos_launch"], diag) < 1e-7
    k = 0
    for c in (1, 30, 90):
        while k < c:
            orc.step()
            k += 1
        tol = H.TOL_1STEP if c == 1 else H.TOL_100STEP
        assert H.max_err_over_diag(orc.positions(), g[f"pos_ground_{c}"], diag) < tol, c
    orc.reset()
    np.testing.assert_array_equal(orc.positions(), g["pos_reset"])
    orc.step()
    assert H.max_err_over_diag(orc.positions(), g["pos_after_reset_step"], diag) < H.TOL_1STEP
    orc.set_ground(False, (0.0, 0.0, 1.0), 0.0, 0.5, 0.3, 0.0, 0.0, 0.0)


def test_rest_is_a_fixed_point(orc):
    """Known answer: with no forces a step at rest moves nothing beyond rounding of the
    rest lengths (the shape goal and the volume dead band are exact fixed points,
    forward.cu:6334, 8602) and the rest J of every volume cluster is 1
    (forward.cu:10370-10397)."""
    sc = H.scenes.make_scene(1500, 21)
    s = H.scenes.Scenario(sc, [])
    s.setup(orc)
    orc.volume_stats(True)
    for _ in range(3):
        orc.step()
    assert H.max_err_over_diag(orc.positions(), sc["pos"], H.scenes.bbox_diagonal(sc["pos"])) < 1e-7
    m, sd = orc.volume_stats(True)
    assert abs(m - 1.0) < 1e-6 and sd < 1e-5


def test_error_behaviour(orc):
    orc.destroy()
    assert orc.lib.xpbd_step() == -1
    assert "create" in orc.last_error()
    sc = H.scenes.make_scene(300, 2)
    rc = orc.lib.xpbd_create(0, sc["pos"].ravel(), sc["scales"].ravel(), sc["rots"].ravel(), sc["opacity"], 0,
                             np.zeros(2, np.int32), np.zeros(1, np.float32), np.zeros(1, np.float32))
    assert rc == -1 and "invalid arguments" in orc.last_error()
    orc.create(sc)
    with pytest.raises(RuntimeError, match="no step yet"):
        orc.positions()
    with pytest.raises(RuntimeError, match="no step yet"):
        orc.set_attached([0], [[0.0, 0.0, 0.0]])
    orc.step()
    with pytest.raises(RuntimeError, match="size mismatch"):
        orc._check(orc.lib.xpbd_positions_host(np.zeros(3, np.float32), 1), "xpbd_positions_host")
    orc.destroy()


def _chainmail_run(solver, sc):
    res = {}

    def record(tag):
        res[tag] = (solver.positions(), solver.chainmail_times())
    H.scenes.chainmail_script(solver, sc, record)
    return res


def test_chainmail_matches_reference(orc):
    """ChainMail waves (runChainmailGPU, forward.cu:12808-13006): arrival times are sums and
    comparisons only, so bit-exact; positions within the 1-step tolerance."""
    g = H.load_golden("chainmail_n4000")
    sc = H.golden_scene(g)
    res = _chainmail_run(orc, sc)
    diag = H.scenes.bbox_diagonal(g["pos_run1"])
    for tag in ("run1", "run2"):
        pos, t = res[tag]
        np.testing.assert_array_equal(t, g[f"time_{tag}"])
        assert H.max_err_over_diag(pos, g[f"pos_{tag}"], diag) < H.TOL_1STEP
    assert (g["time_run1"] < 1e8).sum() > 1000   # the wave travelled


def test_object_mode_two_objects(orc):
    """Object mode on two objects pushed together: rigid fit weighted by the pins, cross-object
    self-collision limited to the other object's box, contact push (forward.cu:12141-12166,
    11796-11849, 12587-12597)."""
    g = H.load_golden("object_blobs")
    s = H.scenario_for("object_blobs")
    s.setup(orc)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    done = 0
    for c in g["checkpoints"]:
        s.advance(orc, int(c) - done)
        done = int(c)
        tol = H.TOL_1STEP if c == 1 else H.TOL_100STEP
        assert H.max_err_over_diag(orc.positions(), g[f"pos_{c}"], diag) < tol, c
        st = orc.self_collision_stats()
        ref = g[f"sc_stats_{c}"]
        assert abs(st[1] - int(ref[1])) <= max(5, 0.01 * int(ref[1])), (c, st, ref)   # active Gaussians
    assert int(g["sc_stats_30"][1]) < len(g["in_pos"])   # the box filter left some out
    orc.set_object_shape(0.0)



SHAPE_CASES = ["plain_n4000", "plain_n4000_fpolar", "object_plain_n4000", "plain_n20000"]


@pytest.mark.parametrize("case", SHAPE_CASES)
def test_deformed_shapes_on_reference_positions(orc, case):
    """The shape writeback (forward.cu:13022-13247) on the positions the reference reached:
    scales within 1e-5 of the bbox diagonal, quaternions within 1e-4 rad wherever the
    principal axes are well defined (relative eigenvalue gap >= 2e-2; the rest, at most a
    tenth, by covariance within 1e-5)."""
    g = H.load_golden(case)
    s = H.scenario_for(case)
    s.setup(orc)
    s.advance(orc, 1)
    last = int(g["checkpoints"][-1])
    orc.set_positions(g[f"pos_{last}"])
    sc_, q_, k_ = orc.shapes(float(g["deform_eps"]))
    assert k_ == int(g["shape_deformed"])
    m = H.shape_parity(sc_, q_, g["shape_scales"], g["shape_quats"], H.scenes.bbox_diagonal(g["in_pos"]))
    assert m["scale"] < H.TOL_1STEP and m["angle"] < 1e-4, m
    assert m["exempt"] < 0.1 and m["cov_exempt"] < 1e-5, m


@pytest.mark.parametrize("case", ["runtime_n4000", "runtime_n4000_ground"])
def test_runtime_scenario(orc, case):
    """The Isaac runtime's configuration and call order (16 iterations at dt 1/60, leader
    spacing 2, 2048-member cap, object shape keeping, ellipsoid contacts, ground with
    gravity and restitution, pads that close, hold and lift): positions at 1e-5 of the
    diagonal after 1 frame and 1e-4 after 10, 30 and 100, collider hits per frame, the
    deformed shapes after the first frame directly and later by covariance."""
    g = H.load_golden(case)
    s = H.runtime_scenario(g)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    got = {}

    def record(solver, frame, shapes):
        got.setdefault("hits", []).append(solver.collider_stats(2)[0])
        if frame in g["checkpoints"]:
            got[frame] = (solver.positions(), shapes)
    assert s.setup(orc)
    s.advance(orc, int(g["checkpoints"][-1]), record)
    np.testing.assert_array_equal(orc.ints("vol_count"), g["vol_count"])
    hits = np.asarray(got["hits"])
    assert np.abs(hits - g["col_hits"]).max() <= 1 and (hits != g["col_hits"]).mean() < 0.05
    for c in g["checkpoints"]:
        pos, (sc_, q_, k_) = got[int(c)]
        tol = H.TOL_1STEP if c == 1 else H.TOL_100STEP
        assert H.max_err_over_diag(pos, g[f"pos_{c}"], diag) < tol, c
        # along the trajectory the 1-ring fit amplifies the positions' differences (a
        # squashed neighbourhood is ill-conditioned): covariances at p99 only
        rel = H.covariance_rel_err(sc_, q_, g[f"shape_scales_{c}"], g[f"shape_quats_{c}"])
        assert np.percentile(rel, 99) < 1e-3, (c, np.percentile(rel, 99))
    # the writeback itself on the positions the reference reached, at every checkpoint
    for c in g["checkpoints"]:
        orc.set_positions(g[f"pos_{c}"])
        sc_, q_, _ = orc.shapes(H.scenes.RuntimeScenario.DEFORM_EPS)
        m = H.shape_parity(sc_, q_, g[f"shape_scales_{c}"], g[f"shape_quats_{c}"], diag)
        assert m["scale"] < H.TOL_1STEP and m["angle"] < 1e-4, (c, m)
        assert m["exempt"] < 0.1 and m["cov_exempt"] < 1e-5, (c, m)


def test_press_harness(orc):
    """Press plates (xpbd_press_*): plate positions, displacement and the 25/50/75/100 %
    settling pauses step for step, positions within the tolerances."""
    g = H.load_golden("press_n3000")
    got = H.press_run(orc, g)
    diag = H.scenes.bbox_diagonal(g["in_pos"])
    for k in g.files:
        if k.startswith("state_"):
            np.testing.assert_allclose(got[k], g[k], rtol=1e-6, atol=1e-6, err_msg=k)
        elif k.startswith("pos_"):
            tol = H.TOL_1STEP if k == "pos_a1" else H.TOL_100STEP
            assert H.max_err_over_diag(got[k], g[k], diag) < tol, k
