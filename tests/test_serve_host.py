"""Host-side logic of the serving loop (no GPU): arena sizing, the scene pool, and the
per-tick collider and pin arrays one arena step call receives."""
import numpy as np

import helpers as H

serve = H.pkg.serve


def test_arena_capacity_respects_budget_and_offsets():
    rows, edges, members, rev = serve.arena_capacity(10e9)
    assert rows * (serve.ARENA_ROW_BYTES + 16 * serve.ARENA_EDGES + 4 * serve.ARENA_MEMBERS
                   + 4 * serve.ARENA_REV) <= 10e9
    assert edges == rows * serve.ARENA_EDGES and members == rows * serve.ARENA_MEMBERS
    rows, edges, members, rev = serve.arena_capacity(150e9)
    assert max(edges, members, rev) <= 2 ** 31 - 1      # 32-bit CSR offsets
    assert serve.arena_bytes(1000) == 1000 * (serve.ARENA_ROW_BYTES + 16 * serve.ARENA_EDGES
                                              + 4 * serve.ARENA_MEMBERS + 4 * serve.ARENA_REV)


def test_scene_pool_stands_in_by_size():
    pool = serve.scene_pool(500, 4000, count=4)
    sizes = [p["pos"].shape[0] for p in pool]
    assert sizes == sorted(sizes) and sizes[0] == 500 and sizes[-1] == 4000
    s = serve.Session(0, 0.0, 1300, 3, 7)
    s.prepare(pool)
    assert s.n == min(sizes, key=lambda v: abs(np.log(v) - np.log(1300)))
    assert s.scen.scene is pool[sizes.index(s.n)]


def test_frame_arrays_cover_every_session():
    pool = serve.scene_pool(500, 2000, count=3)
    sessions = []
    for k, n in enumerate((600, 1500, 2000)):
        s = serve.Session(k, 0.0, n, 4, 11 + k)
        s.prepare(pool)
        s.slot = 10 + k
        s.scen.k = 1 + 10 * k                       # sessions at different frames
        sessions.append(s)
    ty, po, di, cs, ps, pi, tg = serve._frame_arrays(sessions, 10)
    ncol = sum(len(s.scen.grippers) for s in sessions)
    npin = sum(len(g.idx) for s in sessions for g in s.scen.grippers)
    assert ty.shape == (ncol,) and po.shape == (10, ncol, 12) and di.shape == (ncol, 3)
    assert cs.tolist() == [s.slot for s in sessions for _ in s.scen.grippers]
    assert ps.shape == (npin,) and pi.shape == (npin,) and tg.shape == (10, npin, 3)
    # each session's block equals what its own frame call would send
    c0 = p0 = 0
    for s in sessions:
        t1, po1, di1, idx1, tg1 = s.scen.frame_inputs(10)
        k, m = len(t1), len(idx1)
        np.testing.assert_array_equal(po[:, c0:c0 + k], po1)
        np.testing.assert_array_equal(tg[:, p0:p0 + m], tg1)
        np.testing.assert_array_equal(pi[p0:p0 + m], idx1)
        assert (ps[p0:p0 + m] == s.slot).all()
        c0, p0 = c0 + k, p0 + m


def test_pool_sessions_share_the_pinned_set_not_the_motion():
    """Sessions of one pool scene share the gripper's pinned set (computed once per pool
    scene) but keep their own velocity and twist; the inputs equal those of a session
    whose gripper was built from scratch."""
    pool = serve.scene_pool(500, 2000, count=2)
    a = serve.Session(0, 0.0, 2000, 3, 21)
    b = serve.Session(1, 0.0, 2000, 3, 22)
    a.prepare(pool)
    b.prepare(pool)
    ga, gb = a.scen.grippers[0], b.scen.grippers[0]
    assert ga.idx is gb.idx and ga is not gb
    assert not np.array_equal(ga.velocity, gb.velocity) or ga.twist != gb.twist
    own = serve.Session(2, 0.0, 2000, 3, 22)
    own.prepare(list(pool))                            # a plain list: gripper built from scratch
    for x, y in zip(b.scen.frame_inputs(10), own.scen.frame_inputs(10)):
        np.testing.assert_array_equal(x, y)


def test_prefetched_inputs_equal_the_next_frame():
    """The next tick's inputs prepared while the GPU runs the current one are those the
    session's frame call makes when its substep counter arrives there."""
    pool = serve.scene_pool(500, 2000, count=2)
    s = serve.Session(0, 0.0, 1500, 4, 5)
    s.prepare(pool)
    ahead = s.scen.frame_inputs(10, s.scen.k + 10)
    s.scen.k += 10
    for x, y in zip(ahead, s.scen.frame_inputs(10)):
        np.testing.assert_array_equal(x, y)
