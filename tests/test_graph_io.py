"""File formats of the reference pipeline: APGGRPH1 graphs, the renumbered graph .npz,
3DGS PLY, and the runtime's xpbd_create inputs (tools/import_graph.py,
src/xpbd_bridge.py:18-42, forward.cu:4612-4663)."""
import numpy as np

import helpers as H

gio = H.pkg.graph_io


def test_apggrph1_round_trip(tmp_path):
    sc = H.scenes.make_scene(800, 2)
    off, cnt, idx, dist, stiff = gio.scene_csr(sc)
    p = tmp_path / "g.bin"
    gio.write_graph(p, sc["pos"], off, cnt, idx, dist, stiff)
    n, m, g = gio.read_graph(p)
    assert n == 800 and m == 2 * len(sc["edges"])
    np.testing.assert_array_equal(g["pos"], sc["pos"])
    for k, v in zip(("offset", "count", "idx", "dist", "stiff"), (off, cnt, idx, dist, stiff)):
        np.testing.assert_array_equal(g[k], v)


def test_scene_csr_is_load_graph_order():
    """Row i lists i's edges in input order (each edge in both endpoint rows)."""
    sc = H.scenes.make_scene(300, 5)
    off, cnt, idx, dist, _ = gio.scene_csr(sc)
    for i in (0, 7, 150, 299):
        want = [(b if a == i else a, r) for (a, b), r in zip(sc["edges"], sc["rest"]) if i in (a, b)]
        got = list(zip(idx[off[i]:off[i] + cnt[i]], dist[off[i]:off[i] + cnt[i]]))
        assert [(int(a), float(b)) for a, b in got] == [(int(a), float(b)) for a, b in want]


def test_reorder_to_splat_order_and_load_inputs(tmp_path):
    """A graph written in a shuffled (viewer) order renumbers back bit-exactly into the
    splat order, and the runtime inputs rebuilt from PLY + .npz equal the scene."""
    sc = H.scenes.make_scene(1200, 3, opacity=0.7)
    rng = np.random.default_rng(0)
    perm = rng.permutation(1200)                      # viewer node v = splat perm[v]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(1200)
    shuffled = {"pos": sc["pos"][perm], "edges": inv[sc["edges"]], "rest": sc["rest"], "stiff": sc["stiff"]}
    off, cnt, idx, dist, stiff = gio.scene_csr(shuffled)
    gio.write_graph(tmp_path / "w_graph_sibr.bin", shuffled["pos"], off, cnt, idx, dist, stiff)
    _, _, g = gio.read_graph(tmp_path / "w_graph_sibr.bin")
    fields = gio.reorder_graph(g, sc["pos"])
    np.testing.assert_array_equal(fields["sibr_to_usd"], perm)
    gio.save_graph_npz(tmp_path / "w_graph.npz", fields)
    gio.write_ply(tmp_path / "w_crop.ply", gio.splat_fields(sc))
    inp = gio.load_inputs(str(tmp_path), "w")
    np.testing.assert_array_equal(inp["pos"], sc["pos"])
    got = {tuple(e): (r, s) for e, r, s in zip(inp["edges"].tolist(), inp["rest"], inp["stiff"])}
    want = {tuple(sorted(e)): (r, s) for e, r, s in zip(sc["edges"].tolist(), sc["rest"], sc["stiff"])}
    assert got == want
    np.testing.assert_allclose(inp["scales"], sc["scales"], rtol=1e-6)
    np.testing.assert_allclose(inp["opacity"], sc["opacity"], rtol=1e-6)


def test_reorder_rejects_mismatched_positions():
    sc = H.scenes.make_scene(200, 1)
    off, cnt, idx, dist, stiff = gio.scene_csr(sc)
    g = {"pos": sc["pos"], "offset": off, "count": cnt, "idx": idx, "dist": dist, "stiff": stiff}
    other = sc["pos"].copy()
    other[5, 0] = np.nextafter(other[5, 0], np.float32(2))
    import pytest
    with pytest.raises(ValueError):
        gio.reorder_graph(g, other)
