"""Packed weighted edges: {u32 dst, u32 w} stored as one u32
(dst << b | (w - min w)) whenever the bits fit.  Every path must give the
same values with and without packing, files written from a packed graph must
equal the originals byte for byte, and host views must show the original
pairs."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
BLOCK = 64 << 10


@pytest.fixture(scope="module")
def g14w(O):
    g = O.rmat(14, 16)
    return O.CSR(g.off, g.adj, O.weights(g))


def test_packed_layout_and_host_view(T, O, g14w):
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        assert g.esz == 8 and g.mem_esz == 4 and g.weight_bits == 6  # weights 1..64
        off, edges, _ = g.host_arrays()
        assert np.array_equal(edges, g14w.wcsr_edges())
        assert np.array_equal(off, g14w.off)
        g.set_edge_packing(False)
        assert g.mem_esz == 8 and g.weight_bits == 0
        _, edges2, _ = g.host_arrays()
        assert np.array_equal(edges2, g14w.wcsr_edges())
        g.set_edge_packing(True)
        assert g.mem_esz == 4


@pytest.mark.parametrize("frac", [0.0, 0.4, 1.0])
def test_same_values_packed_and_unpacked(T, O, g14w, frac):
    srcs = [1] + O.sources(g14w, 2).tolist()
    want = {s: O.sssp(g14w, s) for s in srcs}
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        for packed in (True, False):
            g.set_edge_packing(packed)
            g.plan(int(frac * g.ne * g.esz), block_bytes=BLOCK)
            for s in srcs:
                for mode in ("scan", "queue"):
                    got, st = g.run("sssp", source=s, compaction=mode, timeout_ms=20000)
                    assert np.array_equal(got, want[s]), (packed, s, mode)
                    got, _ = g.run("bfs", source=s, compaction=mode, timeout_ms=20000)
                    assert np.array_equal(got, O.bfs(g14w, s)), (packed, s, mode)


def test_link_bytes_halve_when_packed(T, O, g14w):
    src = int(O.sources(g14w, 1)[0])  # vertex 1 is isolated at this scale
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        link = {}
        for packed in (True, False):
            g.set_edge_packing(packed)
            g.plan(0, block_bytes=BLOCK)
            _, st = g.run("bfs", source=src, timeout_ms=20000)
            link[packed] = st["link_edge_bytes"]
        assert link[True] * 2 == link[False] > 0


def test_batch_and_serve_packed(T, O, g14w):
    srcs = O.sources(g14w, 24)
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        sums = {}
        for packed in (True, False):
            g.set_edge_packing(packed)
            g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK)
            for algo in ("bfs", "sssp"):
                rows, s, _ = g.batch_run(algo, srcs)
                sums[(packed, algo)] = s
                assert np.array_equal(rows[0], (O.sssp if algo == "sssp" else O.bfs)(g14w, int(srcs[0])))
        for algo in ("bfs", "sssp"):
            assert np.array_equal(sums[(True, algo)], sums[(False, algo)])
        g.set_edge_packing(True)
        g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK)
        with T.Server(g, max_slots=8, timeout_ms=20000) as sv:
            tickets = [(sv.submit(a, int(s)), a, int(s)) for a, s in
                       zip(["sssp", "bfs"] * 4, srcs[:8])]
            for t, a, s in tickets:
                got, qs = sv.wait(t)
                assert np.array_equal(got, (O.sssp if a == "sssp" else O.bfs)(g14w, s)), (a, s)


def test_pagerank_on_packed_weighted_csr(T, O, g14w):
    g14 = O.CSR(g14w.off, g14w.adj)
    want = O.pagerank(g14, 20)
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "csr") as g:
        assert g.weighted and g.mem_esz == 4
        g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK, small_list_degree=1)
        got, _ = g.run("pr_push", pr_iters=20)
        assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-6


@pytest.mark.parametrize("name,fmt,weights", [("toy.wcsr", "wcsr", False),
                                              ("toy_w.csr", "csr", True)])
def test_save_of_packed_graph_is_byte_identical(T, tmp_path, name, fmt, weights):
    src = os.path.join(GOLDEN, name)
    with T.Graph.open(src, fmt, weights=weights) as g:
        assert g.weighted
        out = str(tmp_path / ("copy." + fmt))
        g.save(out)
    assert open(out, "rb").read() == open(src, "rb").read()


def test_wide_weights_stay_unpacked(T, O, g14w):
    rng = np.random.default_rng(7)
    w = rng.integers(1, 1 << 20, size=g14w.ne, dtype=np.uint32)  # 14 + 20 bits > 32
    gw = O.CSR(g14w.off, g14w.adj, w)
    with T.Graph.from_arrays(gw.off, gw.wcsr_edges(), "wcsr") as g:
        assert g.mem_esz == 8 and g.weight_bits == 0
        g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK)
        got, _ = g.run("sssp", source=1, timeout_ms=20000)
        assert np.array_equal(got, O.sssp(gw, 1))
