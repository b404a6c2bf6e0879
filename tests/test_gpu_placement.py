"""Access-driven placement and plan files.

A graph of two disconnected RMAT components (ids 0..n-1 and n..2n-1, so
each component owns its own edge blocks) is queried only inside the second
component.  With tracking on, the blocks of that component report the link
bytes; re-placing by access then keeps exactly those blocks resident and the
same queries read nothing over the link, with identical results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BLOCK = 64 << 10


@pytest.fixture(scope="module")
def two_comp(O):
    a = O.rmat(13, 16)
    n = a.nv
    src, dst = [], []
    for u in range(n):
        for w in a.adj[a.off[u]:a.off[u + 1]]:
            src.append(u)
            dst.append(int(w))
    s = np.array(src, np.int64)
    d = np.array(dst, np.int64)
    return O.from_edges(2 * n, np.concatenate([s, s + n]), np.concatenate([d, d + n])), n


def test_tracking_counts_equal_link_bytes(T, O, two_comp):
    g2, n = two_comp
    with T.Graph.from_arrays(g2.off, g2.adj, "csr") as g:
        g.plan(int(0.3 * g.ne * 4), block_bytes=BLOCK, track_access=True, small_list_degree=1)
        srcs = O.sources(g2, 6)
        link = hbm = 0
        for s in srcs:
            got, st = g.run("bfs", source=int(s), timeout_ms=20000)
            assert np.array_equal(got, O.bfs(g2, int(s)))
            link += st["link_edge_bytes"]
            hbm += st["hbm_edge_bytes"]
        acc = g.block_access()
        vb, res = g.blocks()
        assert int(acc[~res].sum()) == link and int(acc[res].sum()) == hbm


def test_replace_by_access_moves_the_hot_component_into_hbm(T, O, two_comp):
    g2, n = two_comp
    hot = [int(s) for s in O.sources(g2, 200) if s >= n][:6]
    assert hot
    with T.Graph.from_arrays(g2.off, g2.adj, "csr") as g:
        budget = int(0.6 * g.ne * 4)  # the hot component and the boundary block fit
        g.plan(budget, block_bytes=BLOCK, track_access=True, small_list_degree=1,
               policy="prefix")  # prefix keeps the cold first component
        before = [g.run("bfs", source=s, timeout_ms=20000) for s in hot]
        assert sum(st["link_edge_bytes"] for _, st in before) > 0
        g.plan(budget, block_bytes=BLOCK, track_access=True, small_list_degree=1, policy="access")
        after = [g.run("bfs", source=s, timeout_ms=20000) for s in hot]
        for (v0, _), (v1, st) in zip(before, after):
            assert np.array_equal(v0, v1)
        assert sum(st["link_edge_bytes"] for _, st in after) == 0


def test_plan_file_round_trip(T, O, two_comp, tmp_path):
    g2, n = two_comp
    p = str(tmp_path / "g.plan")
    with T.Graph.from_arrays(g2.off, g2.adj, "csr") as g:
        info = g.plan(int(0.35 * g.ne * 4), block_bytes=BLOCK, track_access=True)
        for s in O.sources(g2, 3):
            g.run("bfs", source=int(s), timeout_ms=20000)
        acc = g.block_access()
        vb, res = g.blocks()
        g.save_plan(p)
        g.plan(0, block_bytes=BLOCK)  # something else
        info2 = g.load_plan(p)
        vb2, res2 = g.blocks()
        assert np.array_equal(vb, vb2) and np.array_equal(res, res2)
        assert info2["resident_edge_bytes"] == info["resident_edge_bytes"]
        assert info2["small_list_bytes"] == info["small_list_bytes"]
        s0 = int(O.sources(g2, 1)[0])
        got, _ = g.run("bfs", source=s0, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(g2, s0))
    other = O.rmat(12, 8)
    with T.Graph.from_arrays(other.off, other.adj, "csr") as g:
        with pytest.raises(T.ThvError):
            g.load_plan(p)


def test_server_replans_between_queries(T, O, two_comp):
    g2, n = two_comp
    hot = [int(s) for s in O.sources(g2, 400) if s >= n][:24]
    with T.Graph.from_arrays(g2.off, g2.adj, "csr") as g:
        budget = int(0.6 * g.ne * 4)
        g.plan(budget, block_bytes=BLOCK, track_access=True, small_list_degree=1, policy="prefix")
        _, res0 = g.blocks()
        with T.Server(g, max_slots=8, replan_every=4, timeout_ms=20000) as sv:
            for s in hot:  # one at a time: each runs alone, re-plans in between
                vals, st = sv.wait(sv.submit("bfs", s))
                assert np.array_equal(vals, O.bfs(g2, s))
        vb, res1 = g.blocks()
        hot_blocks = vb[:-1] >= n
        assert res1[hot_blocks].all() and not np.array_equal(res0, res1)
