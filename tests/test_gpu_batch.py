"""Batched multi-source BFS / SSSP: every per-source result equals the
single-source run bit for bit (values and the per-source checksum)."""
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


def sources(O, g, n):
    s = O.sources(g, n).tolist()
    s[0] = 1               # may be isolated: a trivial query in the mix
    s[-1] = s[1]           # duplicate source inside a group
    return np.array(s, np.uint32)


@pytest.mark.parametrize("frac,group", [(0.0, 64), (0.4, 64), (1.0, 64), (0.4, 7), (0.4, 1)])
def test_batched_bfs_equals_single(T, O, g14, frac, group):
    src = sources(O, g14, 70)
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        g.plan(int(frac * g.ne * 4), block_bytes=BLOCK)
        out, sums, st = g.batch_run("bfs", src, group=group, timeout_ms=20000)
        for i, s in enumerate(src):
            want = O.bfs(g14, int(s))
            assert np.array_equal(out[i], want), f"source {s}"
            assert int(sums[i]) == T.values_checksum(want)
        assert st["iterations"] > 0


@pytest.mark.parametrize("frac", [0.0, 0.4, 1.0])
def test_batched_sssp_equals_single(T, O, g14w, frac):
    src = sources(O, g14w, 66)
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        g.plan(int(frac * g.ne * 8), block_bytes=BLOCK)
        out, sums, _ = g.batch_run("sssp", src, timeout_ms=20000)
        for i, s in enumerate(src):
            want = O.sssp(g14w, int(s))
            assert np.array_equal(out[i], want), f"source {s}"
            assert int(sums[i]) == T.values_checksum(want)


def test_sssp_window_options_reach_the_kernel(T, O, g14w):
    """Each call's window and growth must be used even when the launch
    sequence was captured by an earlier call with other options."""
    src = sources(O, g14w, 64)
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK)
        iters = {}
        ref = None
        for delta, growth in [(64, 1), (1, 1), (64, 1), (1, 8), (4, 2)]:
            _, sums, st = g.batch_run("sssp", src, sssp_delta=delta, sssp_growth=growth,
                                      want_values=False, timeout_ms=20000)
            if ref is None:
                ref = sums
            assert np.array_equal(sums, ref), (delta, growth)
            iters[(delta, growth)] = st["iterations"]
        assert iters[(1, 1)] > iters[(1, 8)] and iters[(1, 1)] > iters[(64, 1)]


def test_batched_checksums_only(T, O, g14w):
    src = sources(O, g14w, 64)
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK)
        out, sums, _ = g.batch_run("bfs", src, want_values=False)
        assert out is None
        for i, s in enumerate(src[:8]):
            vals, _ = g.run("bfs", source=int(s))
            assert int(sums[i]) == T.values_checksum(vals)


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
def test_checksum_only_groups_match_single_runs(T, O, g14w, algo):
    """Without output rows the checksums come from a streaming pass over the
    per-source rows; a full group and a partial one (37 of 64 sources) must
    give the single runs' checksums."""
    src = sources(O, g14w, 64 + 37)
    ref = O.sssp if algo == "sssp" else O.bfs
    with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
        g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK)
        out, sums, _ = g.batch_run(algo, src, want_values=False, timeout_ms=20000)
        assert out is None
        for i in sorted(set(range(0, len(src), 9)) | {1, 63, 64, len(src) - 1}):
            assert int(sums[i]) == T.values_checksum(ref(g14w, int(src[i]))), (algo, i)


def test_batched_tuning_is_result_neutral(T, O, g14):
    src = sources(O, g14, 64)
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        g.plan(int(0.4 * g.ne * 4), block_bytes=BLOCK)
        a, sa, _ = g.batch_run("bfs", src)
        b, sb, _ = g.batch_run("bfs", src, small_degree=8, chunk_edges=64)
        assert np.array_equal(a, b) and np.array_equal(sa, sb)


def test_deep_graph_falls_back_to_single_runs(T, O):
    n = 300  # a path deeper than the 254 levels a level byte holds
    c = O.from_edges(n, np.arange(n - 1), np.arange(1, n))
    with T.Graph.from_arrays(c.off, c.adj, "csr") as g:
        g.plan()
        out, sums, _ = g.batch_run("bfs", [0, 5, 299], timeout_ms=20000)
        for i, s in enumerate([0, 5, 299]):
            assert np.array_equal(out[i], O.bfs(c, s))


def test_batch_rejects_bad_input(T, O, g14):
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        with pytest.raises(T.ThvError):
            g.batch_run("bfs", [g14.nv])
        with pytest.raises(T.ThvError):
            g.batch_run("sssp", [1])  # no weights
        with pytest.raises(T.ThvError):
            g.batch_run("cc", [1])


def test_pick_sources_matches_oracle(T, O, g14):
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        assert np.array_equal(g.pick_sources(100), O.sources(g14, 100))


def test_autotuner_picks_and_caches_a_configuration(T, O, g14, tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("THV_TUNE_CACHE", str(cache))
    src = sources(O, g14, 64)
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        g.plan(int(0.4 * g.ne * 4), block_bytes=BLOCK)
        out, sums, _ = g.batch_run("bfs", src, tune=True)
        for i, s in enumerate(src):
            assert np.array_equal(out[i], O.bfs(g14, int(s)))
        line = cache.read_text().strip().splitlines()[-1]
        small, chunk, threads, mid, gsmall, gmid = map(int, line.split("|")[1].split())
        assert threads in (256, 512) and small >= 16 and chunk >= 128
        assert mid >= small and 1 <= gsmall <= 32 and 1 <= gmid <= 32
        assert g.batch_tuned("bfs") == {"small_degree": small, "mid_degree": mid,
                                        "chunk_edges": chunk, "threads": threads,
                                        "small_group": gsmall, "mid_group": gmid, "tuned": 1}
        # cached: a second call reuses it (and still matches)
        out2, sums2, _ = g.batch_run("bfs", src, tune=True)
        assert np.array_equal(sums, sums2)
        assert len(cache.read_text().strip().splitlines()) == 1


def test_direct_launches_equal_graph_replays(T, O, g14w, monkeypatch):
    src = sources(O, g14w, 64)
    res = {}
    for direct in ("0", "1"):
        monkeypatch.setenv("THV_BATCH_DIRECT", direct)
        with T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr") as g:
            g.plan(int(0.4 * g.ne * 8), block_bytes=BLOCK)
            res[direct] = [g.batch_run(a, src, want_values=False, timeout_ms=20000)[1]
                           for a in ("bfs", "sssp")]
    for a, b in zip(res["0"], res["1"]):
        assert np.array_equal(a, b)


@pytest.fixture(scope="module")
def skewed(O):
    """Three degree populations: 40 hubs of out-degree 3000, 1,500 vertices
    of out-degree 120, 18,460 of out-degree 3 (seeded uniform targets)."""
    rng = np.random.default_rng(7)
    nv = 20000
    deg = np.full(nv, 3, np.int64)
    perm = rng.permutation(nv)
    deg[perm[:40]] = 3000
    deg[perm[40:1540]] = 120
    src = np.repeat(np.arange(nv), deg)
    dst = rng.integers(0, nv, len(src))
    g = O.from_edges(nv, src, dst)
    return O.CSR(g.off, g.adj, O.weights(g))


BUCKETS = [
    dict(),                                                   # tuned / default
    dict(small_degree=16, mid_degree=512, chunk_edges=256, small_group=32, mid_group=4),
    dict(small_degree=16, mid_degree=512, chunk_edges=128, small_group=8, mid_group=1),
    dict(small_degree=64, mid_degree=2048, chunk_edges=512, small_group=16, mid_group=2),
    dict(small_degree=16, mid_degree=16, chunk_edges=128, small_group=1),  # two buckets
]


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
def test_degree_buckets_leave_results_unchanged(T, O, skewed, algo, tmp_path, monkeypatch):
    monkeypatch.setenv("THV_TUNE_CACHE", str(tmp_path / "tune.txt"))
    deg = np.diff(skewed.off.astype(np.int64))
    # every bucket of the second configuration is populated
    assert (deg < 16).sum() and ((deg >= 16) & (deg < 512)).sum() and (deg >= 512).sum()
    src = sources(O, skewed, 64)
    want = [O.bfs(skewed, int(s)) if algo == "bfs" else O.sssp(skewed, int(s)) for s in src]
    edges = skewed.adj if algo == "bfs" else skewed.wcsr_edges()
    with T.Graph.from_arrays(skewed.off, edges, "csr" if algo == "bfs" else "wcsr") as g:
        g.plan(int(0.4 * g.ne * g.esz), block_bytes=BLOCK)
        for cfg in BUCKETS:
            out, sums, _ = g.batch_run(algo, src, timeout_ms=20000, **cfg)
            for i, s in enumerate(src):
                assert np.array_equal(out[i], want[i]), f"{cfg} source {s}"
        # tuning times the buckets' settings and reports the one it keeps;
        # the results stay those of the single-source runs
        assert g.batch_tuned(algo)["tuned"] == 0
        out, sums, _ = g.batch_run(algo, src, timeout_ms=20000, tune=True)
        for i, s in enumerate(src):
            assert np.array_equal(out[i], want[i]), f"tuned, source {s}"
        c = g.batch_tuned(algo)
        assert c["tuned"] == 1
        assert 16 <= c["small_degree"] <= c["mid_degree"]
        assert c["threads"] in (256, 512) and c["chunk_edges"] >= 128
        # the buckets get different configurations: grouped vertices share a
        # warp (small_group of them), chunked ones spread over several warps
        assert c["small_group"] >= 1 and c["chunk_edges"] < 3000
        if c["mid_degree"] > c["small_degree"]:
            assert c["mid_group"] < c["small_group"]
