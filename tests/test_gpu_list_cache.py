"""Small-list cache: lists shorter than the plan's threshold that fall in
host blocks are read from a packed HBM copy.  Results stay bit-exact for
every threshold and budget, the plan's byte accounting matches the block
table, and a BFS reads over the host link exactly the lists the cache and
the resident blocks leave there."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BLOCK = 64 << 10


@pytest.fixture(scope="module")
def g14(O):
    return O.rmat(14, 16)


@pytest.fixture(scope="module")
def g14w(O, g14):
    return O.CSR(g14.off, g14.adj, O.weights(g14))


def split(g, csr, info):
    """(cached, host) vertex masks implied by the block table and the plan."""
    vb, res = g.blocks()
    deg = np.diff(csr.off.astype(np.int64))
    blk = np.searchsorted(vb.astype(np.int64), np.arange(len(deg)), side="right") - 1
    host_blk = ~res[blk]
    t = info["small_list_degree"]
    cached = host_blk & (deg > 0) & (deg < t) if t else np.zeros(len(deg), bool)
    return deg, cached, host_blk & ~cached


@pytest.mark.parametrize("deg", [1, 8, 64, 4096])
@pytest.mark.parametrize("frac", [0.25, 0.6])
def test_plan_accounting(T, O, g14, deg, frac):
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        budget = int(frac * g.ne * g.esz)
        info = g.plan(budget, block_bytes=BLOCK, small_list_degree=deg)
        assert info["resident_edge_bytes"] + info["host_edge_bytes"] == g.ne * 4
        assert info["resident_edge_bytes"] <= budget
        if deg == 1:
            assert info["small_list_degree"] == 0 and info["small_list_bytes"] == 0
        else:
            assert 0 < info["small_list_degree"] <= deg
        d, cached, host = split(g, g14, info)
        assert info["small_list_bytes"] == int(d[cached].sum()) * 4
        assert info["small_list_vertices"] == int(cached.sum())
        assert info["host_edge_bytes"] == int(d[host].sum()) * 4


@pytest.mark.parametrize("deg", [1, 8, 64, 4096])
def test_bfs_link_bytes_exact(T, O, g14, deg):
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        info = g.plan(int(0.4 * g.ne * 4), block_bytes=BLOCK, small_list_degree=deg)
        d, cached, host = split(g, g14, info)
        for src in [1] + O.sources(g14, 2).tolist():
            want = O.bfs(g14, src)
            reached = want < g14.nv + 1
            for mode in ("scan", "queue"):
                got, st = g.run("bfs", source=src, compaction=mode, timeout_ms=20000)
                assert np.array_equal(got, want)
                assert st["link_edge_bytes"] == int(d[reached & host].sum()) * 4
                assert st["edges_expanded"] == int(d[reached].sum())


@pytest.mark.parametrize("deg", [8, 64, 4096])
def test_sssp_cc_exact(T, O, g14w, deg):
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK, small_list_degree=deg)
        for src in [1] + O.sources(g14w, 2).tolist():
            want = O.sssp(g14w, src)
            for mode in ("scan", "queue"):
                got, _ = g.run("sssp", source=src, compaction=mode, timeout_ms=20000)
                assert np.array_equal(got, want), (src, mode)
    s = O.rmat(13, 8, symmetric=True)
    with T.Graph.from_arrays(s.off, s.adj, "csr") as g:
        g.plan(int(0.4 * g.ne * 4), block_bytes=BLOCK, small_list_degree=deg)
        want = O.cc(s)
        for mode in ("scan", "queue"):
            got, _ = g.run("cc", compaction=mode, timeout_ms=20000)
            assert np.array_equal(got, want)


def test_batch_and_pagerank_on_cached_plan(T, O, g14w):
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        info = g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK)
        assert info["small_list_bytes"] > 0
        srcs = O.sources(g14w, 40)
        for algo, ref in (("bfs", O.bfs), ("sssp", O.sssp)):
            rows, _, _ = g.batch_run(algo, srcs)
            for i, s in enumerate(srcs[:6]):
                assert np.array_equal(rows[i], ref(g14w, int(s))), (algo, s)
    g14 = O.CSR(g14w.off, g14w.adj)
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        info = g.plan(int(0.4 * g.ne * 4), block_bytes=BLOCK)
        assert info["small_list_bytes"] > 0
        got, _ = g.run("pr_push", pr_iters=20)
        want = O.pagerank(g14, 20)
        assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-6


def test_replan_between_batches(T, O, g14):
    """A re-plan frees the old tables; batched runs must not replay launch
    graphs captured against them."""
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        srcs = O.sources(g14, 8)
        g.plan(int(0.3 * g.ne * 4), block_bytes=BLOCK)
        a, sa, _ = g.batch_run("bfs", srcs)
        g.plan(int(0.7 * g.ne * 4), block_bytes=BLOCK, small_list_degree=1)
        b, sb, _ = g.batch_run("bfs", srcs)
        assert np.array_equal(a, b) and np.array_equal(sa, sb)
        assert np.array_equal(a[0], O.bfs(g14, int(srcs[0])))
