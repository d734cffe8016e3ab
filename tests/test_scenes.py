"""Seeded synthetic workloads: deterministic, and shaped like the reference's inputs."""
import numpy as np

import helpers as H


def test_scene_is_deterministic_and_well_formed():
    a = H.scenes.make_scene(5000, 7)
    b = H.scenes.make_scene(5000, 7)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    e = a["edges"]
    assert e.dtype == np.int32 and (e[:, 0] < e[:, 1]).all()
    assert len(np.unique(e[:, 0].astype(np.int64) * 5000 + e[:, 1])) == len(e)
    deg = np.bincount(e.ravel(), minlength=5000)
    assert deg.min() >= 8            # every node keeps its 8 nearest neighbours
    r = np.asarray(H.scenes.DEFAULT_RADII)
    assert ((a["pos"] / r) ** 2).sum(1).max() <= 1.0 + 1e-5
    np.testing.assert_allclose(np.linalg.norm(a["rots"], axis=1), 1.0, atol=1e-6)
    d = np.linalg.norm(a["pos"][e[:, 0]] - a["pos"][e[:, 1]], axis=1)
    np.testing.assert_allclose(a["rest"], d, rtol=1e-6)


def test_golden_scenes_regenerate_bit_exactly():
    """The committed fixtures were made from these generators."""
    for case in ("plain_n4000", "plain_n20000"):
        g = H.load_golden(case)
        s = H.scenario_for(case)
        np.testing.assert_array_equal(s.scene["pos"], g["in_pos"])
        np.testing.assert_array_equal(s.scene["edges"], g["in_edges"])
        np.testing.assert_array_equal(np.concatenate([gr.idx for gr in s.grippers]), g["pins_idx"])


def test_gripper_motion():
    sc = H.scenes.make_scene(3000, 1)
    gr = H.scenes.Gripper(sc["pos"], (0.9, 0, 0), 50, (0.01, 0, 0), np.radians(1.0))
    t0 = gr.targets(0.0)
    np.testing.assert_allclose(t0, sc["pos"][gr.idx], atol=1e-6)
    t1 = gr.targets(10.0)
    # rigid: pairwise distances preserved
    d0 = np.linalg.norm(t0[:, None] - t0[None], axis=2)
    d1 = np.linalg.norm(t1[:, None] - t1[None], axis=2)
    np.testing.assert_allclose(d0, d1, atol=1e-5)
    typ, pose, dims = gr.collider(10.0)
    assert typ == 2 and pose.shape == (12,) and dims[0] == 0.05


def test_dense_contact_plates_close_then_hold():
    s = H.scenes.dense_contact_scenario(3000, 1)
    assert s.iters == 20 and s.max_members == 128 and s.self_collision
    top, bottom = s.grippers
    z = s.scene["pos"][:, 2]
    thick = float(z.max() - z.min())
    gap = lambda t: (top.centre(t)[2] - top.half[2]) - (bottom.centre(t)[2] + bottom.half[2])
    assert abs(gap(0) - thick) < 1e-6
    assert abs(gap(10) - (thick - 0.05)) < 1e-6            # 0.005 per frame
    assert abs(gap(1000) - 0.4 * thick) < 1e-6             # stops at 40 %
    assert not s.has_pins()
    types, poses, dims = s.colliders(0.0)
    assert list(types) == [1, 1] and poses.shape == (2, 12)

