"""CPU oracle: known answers, self-consistency, generator determinism.

The oracle restates the reference's relaxations (src/bfs/bfs_kernels.cu:4-76,
src/cc/cc_kernels.cu:4-68, src/sssp/sssp_kernels.cu:106-144) with the value
encoding of src/graph.cuh:244-265.
"""
import numpy as np
import pytest


def toy(O, nv, edges):
    s = [e[0] for e in edges]
    d = [e[1] for e in edges]
    return O.from_edges(nv, s, d)


def test_path_bfs_levels(O):
    g = toy(O, 5, [(0, 1), (1, 2), (2, 3), (3, 4)])
    assert O.bfs(g, 0).tolist() == [1, 2, 3, 4, 5]
    assert O.bfs(g, 2).tolist() == [6, 6, 1, 2, 3]  # unreached = n + 1


def test_star_and_unreached(O):
    g = toy(O, 6, [(0, i) for i in range(1, 5)])
    assert O.bfs(g, 0).tolist() == [1, 2, 2, 2, 2, 7]
    assert O.bfs(g, 3).tolist() == [7, 7, 7, 1, 7, 7]


def test_self_loop_and_duplicates_removed(O):
    g = toy(O, 3, [(0, 0), (0, 1), (0, 1), (1, 2), (2, 2)])
    assert g.off.tolist() == [0, 1, 2, 2]
    assert g.adj.tolist() == [1, 2]


def test_cc_min_label_two_components(O):
    g = toy(O, 6, [(0, 1), (1, 0), (1, 2), (2, 1), (4, 5), (5, 4)])
    assert O.cc(g).tolist() == [0, 0, 0, 3, 4, 4]
    assert O.cc(g, parallel=True).tolist() == [0, 0, 0, 3, 4, 4]


def test_cc_directed_is_min_reaching_id(O):
    # reference push semantics on a directed graph: min id of any vertex
    # that reaches v (cc_kernels.cu:58-63)
    g = toy(O, 4, [(3, 0), (0, 1), (2, 1)])
    assert O.cc(g).tolist() == [0, 0, 2, 3]


def test_sssp_known_and_clipped(O):
    g = toy(O, 4, [(0, 1), (1, 2), (0, 2)])
    # off/adj sorted: 0->1, 0->2, 1->2
    g.w = np.array([1, 5, 1], np.uint32)
    assert O.sssp(g, 0).tolist() == [1, 2, 3, 5]
    g.w = np.array([2, 9, 3], np.uint32)  # 1+2+3=6 >= n+1=5 -> clipped
    assert O.sssp(g, 0).tolist() == [1, 3, 5, 5]
    assert O.sssp(g, 0, parallel=True).tolist() == [1, 3, 5, 5]


def test_zero_outdegree_source(O):
    g = toy(O, 3, [(1, 2)])
    assert O.bfs(g, 0).tolist() == [1, 4, 4]


def test_bad_source_raises(O):
    g = toy(O, 3, [(1, 2)])
    with pytest.raises(ValueError):
        O.bfs(g, 3)


def dense_pagerank(nv, edges, iters=20, d=0.85):
    outdeg = np.zeros(nv)
    for s, _ in edges:
        outdeg[s] += 1
    r = np.full(nv, 1.0 / nv)
    for _ in range(iters):
        nxt = np.zeros(nv)
        for s, t in edges:
            nxt[t] += r[s] / outdeg[s]
        dang = r[outdeg == 0].sum()
        r = (1 - d) / nv + d * (nxt + dang / nv)
    return r


def test_pagerank_known(O):
    edges = [(0, 1), (1, 2), (2, 0), (2, 3), (4, 2)]
    g = toy(O, 6, edges)
    want = dense_pagerank(6, sorted(edges))
    got = O.pagerank(g, 20)
    np.testing.assert_allclose(got, want, rtol=1e-13)
    assert abs(got.sum() - 1.0) < 1e-12


@pytest.fixture(scope="module")
def rmat14(O):
    return O.rmat(14, 16)


def test_parallel_matches_sequential(O, rmat14):
    g = rmat14
    for src in O.sources(g, 4):
        assert np.array_equal(O.bfs(g, int(src)), O.bfs(g, int(src), parallel=True))
    assert np.array_equal(O.cc(g), O.cc(g, parallel=True))
    g2 = O.CSR(g.off, g.adj, O.weights(g))
    for src in O.sources(g, 3):
        assert np.array_equal(O.sssp(g2, int(src)), O.sssp(g2, int(src), parallel=True))


def test_pagerank_csr_equals_csc(O, rmat14):
    io, ia, od = O.transpose(rmat14)
    a = O.pagerank(rmat14)
    b = O.pagerank_csc(io, ia, od)
    np.testing.assert_allclose(a, b, rtol=1e-12)
    assert abs(a.sum() - 1.0) < 1e-9


def test_generator_deterministic(O):
    a = O.rmat(12, 8)
    b = O.rmat(12, 8)
    c = O.rmat(12, 8, seed=O.SEED + 1)
    assert np.array_equal(a.off, b.off) and np.array_equal(a.adj, b.adj)
    assert not np.array_equal(a.adj[: min(a.ne, c.ne)], c.adj[: min(a.ne, c.ne)])


def test_generator_properties(O):
    g = O.rmat(12, 16)
    src = np.repeat(np.arange(g.nv, dtype=np.uint64), np.diff(g.off.astype(np.int64)))
    assert (src != g.adj).all()  # no self-loops
    key = src * (1 << 32) + g.adj
    assert (np.diff(key.astype(np.int64)) > 0).all()  # sorted, no duplicates
    assert g.adj.max() < g.nv


def test_permutation_is_bijection(O):
    L = O.lib()
    for scale in (1, 5, 12):
        vals = {L.thvo_permute(x, scale, O.SEED) for x in range(1 << scale)}
        assert vals == set(range(1 << scale))


def test_weights_in_range(O, rmat14):
    w = O.weights(rmat14)
    assert w.min() >= 1 and w.max() <= 64
    assert len(np.unique(w)) == 64


def test_symmetric_graph(O):
    g = O.rmat(11, 8, symmetric=True)
    io, ia, _ = O.transpose(g)
    assert np.array_equal(io, g.off) and np.array_equal(ia, g.adj)


def test_sources_non_isolated(O, rmat14):
    s = O.sources(rmat14, 64)
    deg = np.diff(rmat14.off.astype(np.int64))
    assert (deg[s] > 0).all()
    assert np.array_equal(s, O.sources(rmat14, 64))


def test_source_one_reaches_giant_component_scale20(O):
    g = O.rmat(20, 16)
    lv = O.bfs(g, 1, parallel=True)
    assert O.reached_edges(g, lv) > 0.9 * g.ne
