"""Batched objects and served sessions give each object / session the result it has alone."""
import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

batch = H.pkg.batch
serve = H.pkg.serve


def test_batched_objects_match_alone():
    objs = batch.make_objects(count=4, seed=3, n_min=1500, n_max=4000)
    lib = H.b200()
    b = batch.Batch(objs)
    b.setup(lib)
    b.advance(lib, 20)
    together = b.split(lib.positions())
    for k, (sc, grs) in enumerate(objs):
        s = batch.ObjectScenario(sc, grs)
        s.setup(lib)
        s.advance(lib, 20)
        np.testing.assert_array_equal(lib.positions(), together[k], err_msg=f"object {k}")
    lib.destroy()


def test_engine_instances_are_independent():
    a = H.pkg.bridge.XPBD(H.B200_SO, instance=True)
    b = H.pkg.bridge.XPBD(H.B200_SO, instance=True)
    sa = H.scenes.plain_scene_scenario(2500, 11, pins=20)
    sb = H.scenes.plain_scene_scenario(1800, 12, pins=20)
    sa.setup(a)
    sb.setup(b)
    for _ in range(12):          # interleaved
        sa.advance(a, 1)
        sb.advance(b, 1)
    pa, pb = a.positions(), b.positions()
    a.close()
    b.close()
    c = H.pkg.bridge.XPBD(H.B200_SO, instance=True)
    for s, expect in ((H.scenes.plain_scene_scenario(2500, 11, pins=20), pa),
                      (H.scenes.plain_scene_scenario(1800, 12, pins=20), pb)):
        s.setup(c)
        s.advance(c, 12)
        np.testing.assert_array_equal(c.positions(), expect)
    c.close()


def test_served_sessions_match_alone():
    sessions = [(0.0, 3000, 3, 101), (0.0, 5000, 2, 202), (0.01, 2000, 4, 303)]
    stats = serve.run_served(H.B200_SO, sessions, budget_bytes=1e12)
    assert stats["sessions"] == 3 and stats["steps"] == 9
    done = {s.sid: s for s in stats["sessions_done"]}
    for k, (a, n, frames, seed) in enumerate(sessions):
        alone = serve.Session(k, a, n, frames, seed)
        alone.admit(H.B200_SO)
        while alone.frames_left > 0:
            alone.enqueue_frame()
        alone.solver.lib.xpbd_b200_sync()
        np.testing.assert_array_equal(alone.solver.positions(), done[k].final)
        alone.close(keep_result=False)


def test_served_from_scene_pool_matches_alone():
    """Sessions whose scenes come from a ScenePool join the arena from the pool scene's
    shared prepared engine (two of them from the same one); each session's positions
    equal those of its scene prepared on an engine of its own and stepped alone; the
    plain loop runs the same sessions on the shared engines."""
    pool = serve.scene_pool(2000, 6000, count=2)
    sessions = [(0.0, 2000, 3, 11), (0.0, 6000, 2, 12), (0.005, 2100, 2, 13)]
    stats = serve.run_served(H.B200_SO, sessions, budget_bytes=1e12, pool=pool)
    assert stats["sessions"] == 3 and stats["steps"] == 7
    done = {s.sid: s for s in stats["sessions_done"]}
    for k, (a, n, frames, seed) in enumerate(sessions):
        alone = serve.Session(k, a, n, frames, seed)
        alone.prepare(pool)
        alone.admit(H.B200_SO)
        while alone.frames_left > 0:
            alone.enqueue_frame()
        alone.solver.lib.xpbd_b200_sync()
        np.testing.assert_array_equal(alone.solver.positions(), done[k].final)
        alone.close(keep_result=False)
    plain = serve.run_plain(H.B200_SO, sessions, pool=pool)
    assert plain["sessions"] == 3 and plain["steps"] == 7
    pool.close()


def test_arena_retire_and_compaction_match_alone():
    """Sessions join a small arena, one in the middle retires, a new one only fits after
    the live sessions are moved down over the hole (compaction); every session's
    positions equal its solo run's, bit for bit."""
    specs = {"A": (3000, 101), "B": (5000, 202), "C": (2000, 303), "D": (4000, 404)}

    def session(name):
        n, seed = specs[name]
        s = serve.Session(ord(name), 0.0, n, 99, seed)
        s.admit(H.B200_SO)
        return s

    rows = 11000
    arena = H.pkg.bridge.Arena(H.B200_SO, rows, rows * 12, rows * 66, rows * 68)
    live = {}

    def join(name):
        s = session(name)
        s.slot = arena.admit(s.solver)
        assert s.slot is not None and s.slot >= 0
        s.solver.close()
        live[name] = s

    def tick():
        res = list(live.values())
        arena.step(10, *serve._frame_arrays(res, 10))
        arena.sync()
        for s in res:
            s.scen.k += 10
            s.frames_done = getattr(s, "frames_done", 0) + 1

    for name in "ABC":
        join(name)
    tick()
    tick()
    got = {"B": (arena.positions(live["B"].slot, specs["B"][0]), 2)}
    arena.retire(live.pop("B").slot)
    join("D")                                   # 10,000 rows + 4,000 > 11,000: compaction
    assert arena.usage()["rows"] == 9000
    for _ in range(3):
        tick()
    for name, s in live.items():
        got[name] = (arena.positions(s.slot, s.n), s.frames_done)
    arena.close()
    for name, (pos, frames) in got.items():
        alone = session(name)
        for _ in range(frames):
            alone.enqueue_frame()
        alone.solver.lib.xpbd_b200_sync()
        np.testing.assert_array_equal(alone.solver.positions(), pos, err_msg=name)
        alone.close(keep_result=False)
