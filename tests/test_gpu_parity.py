"""GPU engine vs the CPU oracle (bit-exact; PageRank <= 1e-6 relative).

Every algorithm runs with HBM edge budgets of 0%, 40% and 100% and small
edge blocks, so the zero-copy-only, mixed and fully resident paths all
execute (the reference splits the same work across its static / demand /
filter kernels, src/bfs/bfs.cu:111-519).
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BUDGETS = [0.0, 0.4, 1.0]
BLOCK = 64 << 10  # 64 KiB blocks: many blocks even on small graphs
PR_RTOL = 1e-6    # PageRank: max per-vertex relative error against the FP64 oracle


@pytest.fixture(scope="module")
def g14(O):
    return O.rmat(14, 16)


@pytest.fixture(scope="module")
def g14w(O, g14):
    return O.CSR(g14.off, g14.adj, O.weights(g14))


@pytest.fixture(scope="module")
def g14s(O):
    return O.rmat(14, 8, symmetric=True)


def engine_graph(T, csr, fmt="csr"):
    if fmt == "wcsr":
        return T.Graph.from_arrays(csr.off, csr.wcsr_edges(), "wcsr")
    return T.Graph.from_arrays(csr.off, csr.adj, "csr")


def plan(g, frac, policy="densest"):
    return g.plan(int(frac * g.ne * g.esz), block_bytes=BLOCK, policy=policy)


@pytest.mark.parametrize("frac", BUDGETS)
def test_bfs(T, O, g14, frac):
    with engine_graph(T, g14) as g:
        info = plan(g, frac)
        if frac == 0.0:
            assert info["resident_edge_bytes"] == 0
        if frac == 1.0:
            assert info["host_edge_bytes"] == 0
        for src in [1] + O.sources(g14, 3).tolist():
            got, st = g.run("bfs", source=src, timeout_ms=20000)
            want = O.bfs(g14, src)
            assert np.array_equal(got, want), f"src {src}"
            if st["bottom_up_levels"] == 0:  # bottom-up levels scan in-edges instead
                assert st["edges_expanded"] == O.reached_edges(g14, want)


@pytest.mark.parametrize("frac", BUDGETS)
def test_cc_symmetric(T, O, g14s, frac):
    with engine_graph(T, g14s) as g:
        plan(g, frac, "prefix")
        got, _ = g.run("cc", timeout_ms=20000)
        assert np.array_equal(got, O.cc(g14s))


def test_cc_directed(T, O, g14):
    with engine_graph(T, g14) as g:
        plan(g, 0.4)
        got, _ = g.run("cc", timeout_ms=20000)
        assert np.array_equal(got, O.cc(g14))


@pytest.mark.parametrize("frac", BUDGETS)
def test_sssp_wcsr(T, O, g14w, frac):
    with engine_graph(T, g14w, "wcsr") as g:
        plan(g, frac)
        for src in [1] + O.sources(g14w, 2).tolist():
            got, _ = g.run("sssp", source=src, timeout_ms=20000)
            assert np.array_equal(got, O.sssp(g14w, src)), f"src {src}"


@pytest.mark.parametrize("delta", [1, 7, 100000])
def test_sssp_delta_independent(T, O, g14w, delta):
    src = int(O.sources(g14w, 1)[0])
    with engine_graph(T, g14w, "wcsr") as g:
        plan(g, 0.4)
        got, _ = g.run("sssp", source=src, sssp_delta=delta, timeout_ms=20000)
        assert np.array_equal(got, O.sssp(g14w, src))


@pytest.mark.parametrize("growth", [1, 2, 8, 1 << 20])
@pytest.mark.parametrize("mode", ["scan", "queue"])
def test_sssp_growth_independent(T, O, g14w, growth, mode):
    src = int(O.sources(g14w, 1)[0])
    with engine_graph(T, g14w, "wcsr") as g:
        plan(g, 0.4)
        for delta in (1, 8):
            got, _ = g.run("sssp", source=src, sssp_delta=delta, sssp_growth=growth,
                           compaction=mode, timeout_ms=20000)
            assert np.array_equal(got, O.sssp(g14w, src)), (delta, growth, mode)


@pytest.mark.parametrize("small,chunk", [(1, 32), (32, 64), (1024, 1024)])
def test_expansion_tuning_is_result_neutral(T, O, g14, small, chunk):
    with engine_graph(T, g14) as g:
        plan(g, 0.4)
        got, _ = g.run("bfs", source=1, small_degree=small, chunk_edges=chunk, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(g14, 1))
        got, _ = g.run("cc", small_degree=small, chunk_edges=chunk, timeout_ms=20000)
        assert np.array_equal(got, O.cc(g14))


def max_rel(got, want):
    return float(np.max(np.abs(got - want) / np.abs(want)))


@pytest.mark.parametrize("frac", BUDGETS)
def test_pagerank_push(T, O, g14, frac):
    want = O.pagerank(g14, 20)
    with engine_graph(T, g14) as g:
        plan(g, frac)
        got, st = g.run("pr_push", pr_iters=20)
        assert got.dtype == np.float64
        assert max_rel(got, want) <= PR_RTOL
        assert st["edges_expanded"] == 20 * g14.ne


@pytest.mark.parametrize("frac", BUDGETS)
def test_pagerank_pull(T, O, g14, frac):
    io, ia, od = O.transpose(g14)
    want = O.pagerank_csc(io, ia, od, 20)
    with T.Graph.from_arrays(io, ia, "csc", outdeg=od) as g:
        plan(g, frac)
        got, _ = g.run("pr_pull", pr_iters=20)
        assert max_rel(got, want) <= PR_RTOL


@pytest.mark.parametrize("frac", [0.0, 0.4])
def test_pagerank_scale20_twenty_iterations_every_vertex(T, O, frac):
    # config-3 shape at scale 20 (1 M vertices, 16 M edges, hub in-degrees in
    # the thousands): pull over the CSC and push over the CSR of the same
    # graph, 20 iterations, every vertex against one FP64 oracle run, with
    # part (or none) of the edges resident and the rest read over the link
    g = O.rmat(20, 16)
    io, ia, od = O.transpose(g)
    want = O.pagerank_csc(io, ia, od, 20)
    with T.Graph.from_arrays(io, ia, "csc", outdeg=od) as eg:
        eg.plan(int(frac * eg.ne * 4), small_list_degree=1)
        got, _ = eg.run("pr_pull", pr_iters=20)
        assert max_rel(got, want) <= PR_RTOL
    with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
        eg.plan(int(frac * eg.ne * 4), small_list_degree=1)
        got, _ = eg.run("pr_push", pr_iters=20)
        assert max_rel(got, want) <= PR_RTOL


def test_pagerank_hub_split_tiles(T, O):
    # one vertex with in/out-degree 20000 (> tile size): split tiles
    n = 30000
    src = np.concatenate([np.zeros(20000), np.arange(1, 20001), np.arange(100, 5000)])
    dst = np.concatenate([np.arange(1, 20001), np.zeros(20000), np.arange(101, 5001)])
    c = O.from_edges(n, src.astype(np.uint32), dst.astype(np.uint32))
    want = O.pagerank(c, 20)
    with engine_graph(T, c) as g:
        plan(g, 0.5)
        got, _ = g.run("pr_push")
        assert max_rel(got, want) <= PR_RTOL
    io, ia, od = O.transpose(c)
    with T.Graph.from_arrays(io, ia, "csc", outdeg=od) as g:
        plan(g, 0.5)
        got, _ = g.run("pr_pull")
        assert max_rel(got, want) <= PR_RTOL
    with engine_graph(T, c) as g:
        plan(g, 0.3)
        got, _ = g.run("bfs", source=0, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(c, 0))


TOYS = {
    "path": (6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5)]),
    "star": (9, [(0, i) for i in range(1, 8)]),
    "two_components": (7, [(0, 1), (1, 0), (1, 2), (2, 1), (4, 5), (5, 4), (5, 6), (6, 5)]),
    "self_loop_dup": (4, [(0, 0), (0, 1), (0, 1), (1, 2), (2, 3), (3, 3)]),
    "zero_outdeg": (3, [(1, 2), (2, 1)]),
    "single": (1, []),
}


@pytest.mark.parametrize("name", sorted(TOYS))
def test_toy_graphs(T, O, name):
    nv, edges = TOYS[name]
    c = O.from_edges(nv, [e[0] for e in edges], [e[1] for e in edges])
    c.w = (np.arange(c.ne, dtype=np.uint32) % 5) + 1
    with engine_graph(T, c, "wcsr") as g:
        plan(g, 0.5)
        for src in range(nv):
            got, _ = g.run("bfs", source=src, timeout_ms=10000)
            assert np.array_equal(got, O.bfs(c, src))
            got, _ = g.run("sssp", source=src, timeout_ms=10000)
            assert np.array_equal(got, O.sssp(c, src))
        got, _ = g.run("cc", timeout_ms=10000)
        assert np.array_equal(got, O.cc(c))


def test_bad_source(T, O, g14):
    with engine_graph(T, g14) as g:
        with pytest.raises(T.ThvError) as e:
            g.run("bfs", source=g14.nv)
        assert e.value.status == T.THV_EINVAL


def test_wrong_format_errors(T, O, g14):
    with engine_graph(T, g14) as g:
        with pytest.raises(T.ThvError):
            g.run("sssp", source=1)  # no weights
        with pytest.raises(T.ThvError):
            g.run("pr_pull")  # needs CSC


@pytest.mark.parametrize("fmt,sym", [("csr", False), ("wcsr", False), ("csc", False), ("csr", True)])
def test_gpu_generator_matches_oracle(T, O, fmt, sym):
    scale, ef = 13, 16
    want = O.rmat(scale, ef, symmetric=sym)
    with T.Graph.generate_rmat(scale, ef, symmetric=sym, fmt=fmt) as g:
        off, edges, outdeg = g.host_arrays()
        if fmt == "csc":
            io, ia, od = O.transpose(want)
            assert np.array_equal(off, io) and np.array_equal(edges, ia)
            assert np.array_equal(outdeg, od)
        elif fmt == "wcsr":
            assert np.array_equal(off, want.off)
            assert np.array_equal(edges[:, 0], want.adj)
            assert np.array_equal(edges[:, 1], O.weights(want))
        else:
            assert np.array_equal(off, want.off) and np.array_equal(edges, want.adj)


def test_open_files_and_save_roundtrip(T, O, g14w, tmp_path):
    p = str(tmp_path / "g.csr")
    O.write_csr(p, g14w)
    with T.Graph.open(p, "csr", weights=True) as g:
        off, edges, _ = g.host_arrays()
        assert np.array_equal(off, g14w.off)
        assert np.array_equal(edges[:, 0], g14w.adj) and np.array_equal(edges[:, 1], g14w.w)
        got, _ = g.run("sssp", source=1)
        assert np.array_equal(got, O.sssp(g14w, 1))
        q = str(tmp_path / "h.csr")
        g.save(q)
        assert open(q, "rb").read() == open(p, "rb").read()
    p2 = str(tmp_path / "g.wcsr")
    O.write_wcsr(p2, g14w)
    with T.Graph.open(p2, "wcsr") as g:
        got, _ = g.run("sssp", source=1)
        assert np.array_equal(got, O.sssp(g14w, 1))


def test_golden_converter_files_load(T, root):
    gold = os.path.join(root, "tests", "golden")
    for name, fmt, w in [("toy.csr", "csr", False), ("toy_w.csr", "csr", True),
                         ("toy.wcsr", "wcsr", False), ("toy.csc", "csc", False)]:
        with T.Graph.open(os.path.join(gold, name), fmt, weights=w) as g:
            b = open(os.path.join(gold, name), "rb").read()
            nv, ne = np.frombuffer(b[:16], np.uint64)
            assert g.nv == nv and g.ne == ne


def test_cli_end_to_end(T, O, root, g14w, tmp_path):
    p = str(tmp_path / "g.csr")
    O.write_csr(p, g14w)
    os.makedirs(tmp_path / "results")
    for algo, want in [("bfs", O.bfs(g14w, 1)), ("cc", O.cc(g14w)), ("sssp", O.sssp(g14w, 1))]:
        r = subprocess.run([os.path.join(root, "main"), "--input", p, "--algo", algo, "--runs", "2",
                            "--hbm-budget", "40%", "--block-bytes", "64K"],
                           capture_output=True, text=True, cwd=tmp_path, timeout=120)
        assert r.returncode == 0, r.stderr
        assert "Average execution time" in r.stdout
        got = np.fromfile(tmp_path / "results" / "values.bin", np.uint32)
        assert np.array_equal(got, want), algo
    pc = str(tmp_path / "g.csc")
    O.write_csc(pc, g14w)
    r = subprocess.run([os.path.join(root, "main"), "--input", pc, "--algo", "pr", "--type", "pull"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "results" / "values.bin", np.float64)
    assert max_rel(got, O.pagerank(g14w, 20)) <= PR_RTOL


def test_reference_named_drivers(T, O, g14w, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    os.makedirs("results")
    p = str(tmp_path / "g.csr")
    O.write_csr(p, g14w)
    vals, avg = T.BFS32(p, 1, 2)
    assert np.array_equal(vals, O.bfs(g14w, 1)) and avg > 0
    assert np.array_equal(np.fromfile("results/values.bin", np.uint32), vals)
    vals, _ = T.SSSP32(p, 1, 1)
    assert np.array_equal(vals, O.sssp(g14w, 1))
    vals, _ = T.CC32(p, 1)
    assert np.array_equal(vals, O.cc(g14w))
    vals, _ = T.PR32_PUSH(p, 1)
    assert max_rel(vals, O.pagerank(g14w, 20)) <= PR_RTOL


def test_run_checksum_flag(T, O, g14):
    with engine_graph(T, g14) as g:
        plan(g, 0.4)
        vals, st = g.run("bfs", source=1, checksum=True)
        assert st["checksum"] == T.values_checksum(vals)


@pytest.mark.parametrize("frac", [0.0, 0.4])
def test_scan_and_queue_compaction_agree(T, O, g14w, frac):
    """Both work-queue constructions (bitmap scan every iteration, or
    queueing vertices as they are lowered) give the oracle's values."""
    with engine_graph(T, g14w, "wcsr") as g:
        plan(g, frac)
        for src in O.sources(g14w, 2).tolist():
            for mode in ("scan", "queue"):
                got, _ = g.run("bfs", source=src, compaction=mode, timeout_ms=20000)
                assert np.array_equal(got, O.bfs(g14w, src))
                got, _ = g.run("sssp", source=src, compaction=mode, timeout_ms=20000)
                assert np.array_equal(got, O.sssp(g14w, src))
        for mode in ("scan", "queue"):
            got, _ = g.run("cc", compaction=mode, timeout_ms=20000)
            assert np.array_equal(got, O.cc(g14w))


def test_bfs_direction_optimising(T, O, g14):
    """All edges resident: BFS switches to bottom-up levels over the in-edge
    transpose for large frontiers; values equal the top-down run's."""
    srcs = O.sources(g14, 4).tolist()
    with engine_graph(T, g14) as g:
        plan(g, 1.0)
        used = 0
        for s in srcs:
            want = O.bfs(g14, s)
            got, st = g.run("bfs", source=s, timeout_ms=20000)
            assert np.array_equal(got, want), s
            used += st["bottom_up_levels"]
            td, st_td = g.run("bfs", source=s, top_down_only=True, timeout_ms=20000)
            assert np.array_equal(td, want) and st_td["bottom_up_levels"] == 0
            assert st_td["edges_expanded"] == O.reached_edges(g14, want)
        assert used > 0
        plan(g, 0.4)  # host blocks: no transpose, top-down only
        _, st = g.run("bfs", source=srcs[0], timeout_ms=20000)
        assert st["bottom_up_levels"] == 0


def test_bfs_direction_optimising_symmetric_and_toys(T, O):
    s = O.rmat(13, 8, symmetric=True)
    with engine_graph(T, s) as g:
        plan(g, 1.0)
        for src in O.sources(s, 3).tolist():
            got, _ = g.run("bfs", source=src, timeout_ms=20000)
            assert np.array_equal(got, O.bfs(s, src))
    # a star whose centre reaches everything in one level, then a path
    n = 2000
    src_ = [0] * (n - 1) + list(range(1, n - 1))
    dst_ = list(range(1, n)) + list(range(2, n))
    t = O.from_edges(n, src_, dst_)
    with engine_graph(T, t) as g:
        plan(g, 1.0)
        got, _ = g.run("bfs", source=0, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(t, 0))


def _upper_edges(csr):
    off = csr.off.astype(np.int64)
    u = np.repeat(np.arange(csr.nv), np.diff(off))
    return int((csr.adj.astype(np.int64) > u).sum())


@pytest.mark.parametrize("frac", BUDGETS)
def test_cc_union_find_on_symmetric_graphs(T, O, g14s, frac):
    """Marked symmetric: CC runs as sampling union-find, reads far fewer
    edges and returns the min-label fixed point."""
    want = O.cc(g14s)
    with engine_graph(T, g14s) as g:
        assert g.sorted and not g.symmetric
        plan(g, frac)
        lp, st_lp = g.run("cc", timeout_ms=20000)
        g.set_symmetric(True)
        uf, st_uf = g.run("cc", timeout_ms=20000)
        assert np.array_equal(lp, want) and np.array_equal(uf, want)
        assert st_uf["edges_expanded"] < _upper_edges(g14s) < st_lp["edges_expanded"]
        lp2, _ = g.run("cc", label_propagation=True, timeout_ms=20000)
        assert np.array_equal(lp2, want)


def test_cc_union_find_generated_weighted_and_unsorted(T, O):
    # generated symmetric graphs are marked symmetric and sorted
    g = T.Graph.generate_rmat(13, 8, symmetric=True, fmt="wcsr")
    assert g.symmetric and g.sorted and g.mem_esz == 4
    s = O.rmat(13, 8, symmetric=True, weighted=True)
    g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK)
    got, st = g.run("cc", timeout_ms=20000)
    assert np.array_equal(got, O.cc(s)) and st["edges_expanded"] < _upper_edges(s)
    g.close()
    # unsorted lists: the sample is any two neighbours; labels stay exact
    rng = np.random.default_rng(5)
    sym = O.rmat(12, 8, symmetric=True)
    adj = sym.adj.copy()
    for v in range(sym.nv):
        a, b = int(sym.off[v]), int(sym.off[v + 1])
        adj[a:b] = rng.permutation(adj[a:b])
    with T.Graph.from_arrays(sym.off, adj, "csr") as g2:
        g2.set_symmetric(True)
        assert not g2.sorted
        g2.plan(int(0.4 * g2.ne * 4), block_bytes=BLOCK)
        got, st = g2.run("cc", timeout_ms=20000)
        assert np.array_equal(got, O.cc(sym))


def test_cc_union_find_many_components_and_toys(T, O):
    """Components of every size, isolated vertices and a hub outside the
    largest component: the sampled hub component must not hide edges."""
    rng = np.random.default_rng(9)
    parts, base = [], 0
    for size in [1, 2, 3, 50, 400, 3000, 1, 7]:
        if size > 1:
            n_e = size * 3
            s = rng.integers(0, size, n_e) + base
            d = rng.integers(0, size, n_e) + base
            parts.append((s, d))
        base += size
    # a star whose centre (highest degree) is a small component of its own
    hub = base
    leaves = np.arange(base + 1, base + 120)
    parts.append((np.full(len(leaves), hub), leaves))
    base += 120
    s = np.concatenate([p[0] for p in parts])
    d = np.concatenate([p[1] for p in parts])
    g = O.from_edges(base, s, d, symmetric=True)
    with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
        eg.set_symmetric(True)
        for frac in (0.0, 1.0):
            eg.plan(int(frac * eg.ne * 4), block_bytes=BLOCK)
            got, _ = eg.run("cc", timeout_ms=20000)
            assert np.array_equal(got, O.cc(g)), frac
