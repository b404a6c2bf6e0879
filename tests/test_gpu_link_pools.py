"""Host-list chunk pools and small-phase splitting against the CPU oracle.

Queue and scan mode keep chunks of lists read over the host link in their
own pool (the top of the chunk queue), drained first by one warp in six;
queue mode sends every host-read list to that pool whatever its degree,
and splits chunk items into parts in phases with fewer tasks than warps.
These tests drive the extremes: no small-list cache (so every host list,
down to degree 1, becomes a chunk item and the chunk-queue capacity must
count them), no HBM budget at all (every chunk in the host pool), re-plans
between cache on and off on one graph (the run state is re-sized), and
graphs small enough that most phases split their chunks.  Results must be
bit-exact whatever the pools and splits (the relaxation's fixed point is
unique).  Reference: the static/demand split these pools replace,
src/bfs/bfs.cu:111-519 and src/sssp/sssp.cu:10-570.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BLOCK = 16 << 10  # small edge blocks: host and HBM blocks interleave


@pytest.fixture(scope="module")
def g16(O):
    return O.rmat(16, 16)


@pytest.fixture(scope="module")
def g16w(O, g16):
    return O.CSR(g16.off, g16.adj, O.weights(g16))


@pytest.mark.parametrize("budget", [0.0, 0.15, 0.5])
def test_sssp_every_host_list_as_chunks(T, O, g16w, budget):
    srcs = [int(s) for s in O.sources(g16w, 3)]
    want = {s: O.sssp(g16w, s) for s in srcs}
    with T.Graph.from_arrays(g16w.off, g16w.wcsr_edges(), "wcsr") as g:
        # no small-list cache: host lists of every degree are chunk items
        # (budgets in stored bytes: packed weighted edges take 4 bytes)
        g.plan(int(budget * g.ne * g.mem_esz), block_bytes=BLOCK, small_list_degree=1)
        for s in srcs:
            got, st = g.run("sssp", source=s)
            assert np.array_equal(got, want[s]), s
            if budget < 1.0:
                assert st["link_edge_bytes"] > 0
        # the cache back on: fewer chunk items, the same answers
        g.plan(int(budget * g.ne * g.mem_esz), block_bytes=BLOCK)
        for s in srcs:
            assert np.array_equal(g.run("sssp", source=s)[0], want[s]), s
        # and off again after it (the chunk queue grows back)
        g.plan(int(budget * g.ne * g.mem_esz), block_bytes=BLOCK, small_list_degree=1)
        assert np.array_equal(g.run("sssp", source=srcs[0])[0], want[srcs[0]])


@pytest.mark.parametrize("algo", ["bfs", "cc"])
@pytest.mark.parametrize("compaction", ["queue", "scan"])
def test_bfs_cc_pools_without_list_cache(T, O, g16, algo, compaction):
    s = int(O.sources(g16, 1)[0])
    want = O.bfs(g16, s) if algo == "bfs" else O.cc(g16)
    with T.Graph.from_arrays(g16.off, g16.adj, "csr") as g:
        for budget in (0.0, 0.3):
            g.plan(int(budget * g.ne * 4), block_bytes=BLOCK, small_list_degree=1)
            kw = {"label_propagation": True} if algo == "cc" else {"top_down_only": True}
            got, _ = g.run(algo, source=s, compaction=compaction, **kw)
            assert np.array_equal(got, want), budget


@pytest.mark.parametrize("small_degree", [16, 64, 256, 1024])
def test_sssp_small_degree_and_tiny_graph_phases(T, O, small_degree):
    # scale 10: every phase has fewer tasks than warps, so chunk items are
    # split into parts and groups shrink; the group bound varies the mix of
    # groups and chunks
    g = O.rmat(10, 16)
    gw = O.CSR(g.off, g.adj, O.weights(g))
    srcs = [int(x) for x in O.sources(g, 4)]
    with T.Graph.from_arrays(gw.off, gw.wcsr_edges(), "wcsr") as eg:
        eg.plan(int(0.3 * eg.ne * eg.esz), block_bytes=16 << 10)
        for s in srcs:
            got, _ = eg.run("sssp", source=s, small_degree=small_degree)
            assert np.array_equal(got, O.sssp(gw, s)), (s, small_degree)
