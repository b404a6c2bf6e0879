"""Serving: continuous batching.  Every query's result equals the single
-source run bit for bit, whether it ran alone, started a batched group,
joined a batched group already on the device (into a freed mask bit), or
joined a slot traversal mid-stream."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g14w(O):
    g = O.rmat(14, 16)
    return O.CSR(g.off, g.adj, O.weights(g))


@pytest.fixture(scope="module")
def eg(T, g14w):
    g = T.Graph.from_arrays(g14w.off, g14w.wcsr_edges(), "wcsr")
    g.plan(int(0.4 * g.ne * 8), block_bytes=64 << 10)
    yield g
    g.close()


def want(O, g, algo, s):
    return O.bfs(g, s) if algo == "bfs" else O.sssp(g, s)


def test_serve_mixed_stream(T, O, g14w, eg):
    src = O.sources(g14w, 48).tolist() + [1]
    algos = ["sssp" if i % 5 == 0 else "bfs" for i in range(len(src))]
    with T.Server(eg, max_slots=8, timeout_ms=20000) as sv:
        tickets = [sv.submit(a, s) for a, s in zip(algos, src)]
        for t, a, s in zip(tickets, algos, src):
            vals, st = sv.wait(t)
            w = want(O, g14w, a, s)
            assert np.array_equal(vals, w), f"{a} {s}"
            assert st["checksum"] == T.values_checksum(w)
            assert st["status"] == 0 and st["latency_ms"] >= st["run_ms"]


def test_serve_arrivals_join_running_traversal(T, O, g14w, eg):
    src = O.sources(g14w, 24).tolist()
    with T.Server(eg, max_slots=4, max_batch_iters=1, group_min=0xFFFFFFFF,
                  timeout_ms=20000) as sv:
        tickets = []
        for i, s in enumerate(src):
            tickets.append((sv.submit("sssp" if i % 3 == 0 else "bfs", s), s, i))
            time.sleep(0.0005 * (i % 4))
        slots = set()
        for t, s, i in tickets:
            vals, st = sv.wait(t)
            slots.add(st["slot"])
            assert np.array_equal(vals, want(O, g14w, "sssp" if i % 3 == 0 else "bfs", s))
        assert slots <= set(range(4))


def test_serve_same_result_alone_and_in_mix(T, O, g14w, eg):
    s0 = int(O.sources(g14w, 1)[0])
    with T.Server(eg, max_slots=1) as sv:
        alone, st_a = sv.wait(sv.submit("sssp", s0))
    with T.Server(eg, max_slots=16, group_min=0xFFFFFFFF) as sv:
        ts = [sv.submit("bfs", s) for s in O.sources(g14w, 10)]
        t0 = sv.submit("sssp", s0)
        ts += [sv.submit("bfs", s) for s in O.sources(g14w, 20)[10:]]
        mixed, st_m = sv.wait(t0)
        for t in ts:
            sv.wait(t)
    assert np.array_equal(alone, mixed) and st_a["checksum"] == st_m["checksum"]


def test_serve_memory_admission(T, O, g14w, eg):
    per_slot = eg.nv * 4
    with T.Server(eg, max_slots=64, mem_budget_bytes=3 * per_slot) as sv:
        ts = [(sv.submit("bfs", s), s) for s in O.sources(g14w, 12)]
        used = set()
        for t, s in ts:
            vals, st = sv.wait(t)
            used.add(st["slot"])
            assert np.array_equal(vals, O.bfs(g14w, s))
        assert used <= {0, 1, 2}
    with pytest.raises(T.ThvError) as e:
        T.Server(eg, mem_budget_bytes=per_slot - 1)
    assert e.value.status == T.THV_ENOMEM


def test_serve_checksum_only_and_poll(T, O, g14w, eg):
    with T.Server(eg) as sv:
        t = sv.submit("bfs", int(O.sources(g14w, 1)[0]), want_values=False)
        res = None
        for _ in range(20000):
            res = sv.poll(t)
            if res is not None:
                break
            time.sleep(0.001)
        vals, st = res
        assert vals is None
        assert st["checksum"] == T.values_checksum(O.bfs(g14w, int(O.sources(g14w, 1)[0])))


def test_serve_rejects_bad_requests(T, O, g14w, eg):
    with T.Server(eg) as sv:
        with pytest.raises(T.ThvError):
            sv.submit("bfs", eg.nv)
        with pytest.raises(T.ThvError):
            sv.submit("cc", 1)
    gu = T.Graph.from_arrays(g14w.off, g14w.adj, "csr")
    with T.Server(gu) as sv:
        with pytest.raises(T.ThvError):
            sv.submit("sssp", 1)
    gu.close()


def test_deep_queue_runs_as_batched_groups(T, O, g14w, eg):
    src = O.sources(g14w, 100).tolist()
    algos = ["sssp" if i % 4 == 0 else "bfs" for i in range(len(src))]
    with T.Server(eg, max_slots=8, group_min=16, timeout_ms=20000) as sv:
        tickets = [sv.submit(a, s, want_values=(i % 2 == 0)) for i, (a, s) in
                   enumerate(zip(algos, src))]
        grouped = 0
        for i, (t, a, s) in enumerate(zip(tickets, algos, src)):
            vals, st = sv.wait(t)
            w = want(O, g14w, a, s)
            assert st["checksum"] == T.values_checksum(w), f"{a} {s}"
            if i % 2 == 0:
                assert np.array_equal(vals, w), f"{a} {s}"
            grouped += st["grouped"]
        assert grouped > 0


def test_group_mode_can_be_switched_off(T, O, g14w, eg):
    src = O.sources(g14w, 60).tolist()
    with T.Server(eg, max_slots=4, group_min=0xFFFFFFFF, timeout_ms=20000) as sv:
        tickets = [(sv.submit("bfs", s), s) for s in src]
        for t, s in tickets:
            vals, st = sv.wait(t)
            assert st["grouped"] != 1 and st["slot"] < 4
            assert np.array_equal(vals, O.bfs(g14w, s))


def test_idle_server_runs_a_lone_query_on_the_single_source_kernel(T, O, g14w, eg):
    s0 = int(O.sources(g14w, 1)[0])
    with T.Server(eg, max_slots=8, timeout_ms=20000) as sv:
        for algo in ("bfs", "sssp"):
            vals, st = sv.wait(sv.submit(algo, s0))
            assert st["grouped"] == 2
            assert np.array_equal(vals, want(O, g14w, algo, s0))
            assert st["checksum"] == T.values_checksum(vals)


@pytest.mark.parametrize("group_min", [0, 16, 0xFFFFFFFF])
def test_all_serving_modes_agree(T, O, g14w, eg, group_min):
    src = O.sources(g14w, 40).tolist()
    algos = ["sssp" if i % 3 == 0 else "bfs" for i in range(len(src))]
    with T.Server(eg, max_slots=8, group_min=group_min, timeout_ms=20000) as sv:
        tickets = [sv.submit(a, s, want_values=False) for a, s in zip(algos, src)]
        modes = set()
        for t, a, s in zip(tickets, algos, src):
            _, st = sv.wait(t)
            modes.add(st["grouped"])
            assert st["checksum"] == T.values_checksum(want(O, g14w, a, s)), (a, s)
        if group_min == 0xFFFFFFFF:
            assert 1 not in modes


def graph_with_tail(O, T, tail, seed_scale=14):
    """RMAT plus a path of `tail` vertices hanging off its highest-degree
    vertex: traversals that reach the hub last about `tail` iterations, so a
    batched group stays on the device long enough for arrivals to join."""
    g = O.rmat(seed_scale, 16)
    deg = np.diff(g.off.astype(np.int64))
    hub = int(np.argmax(deg))
    src = np.repeat(np.arange(g.nv, dtype=np.uint32), deg)
    path = np.arange(g.nv, g.nv + tail, dtype=np.uint32)
    s = np.concatenate([src, [hub], path[:-1]]).astype(np.uint32)
    d = np.concatenate([g.adj, [g.nv], path[1:]]).astype(np.uint32)
    gp = O.from_edges(g.nv + tail, s, d)
    gp = O.CSR(gp.off, gp.adj, O.weights(gp))
    eg = T.Graph.from_arrays(gp.off, gp.wcsr_edges(), "wcsr")
    eg.plan(int(0.4 * eg.ne * 8), block_bytes=64 << 10)
    return gp, eg, hub


@pytest.mark.parametrize("algo,tail", [("sssp", 6000), ("bfs", 100)])
def test_arrival_joins_a_running_batched_group(T, O, algo, tail):
    # group_min 1: the first query starts a batched group at once; with the
    # join window open for the group's whole life, queries submitted while
    # it runs must join it mid-flight (grouped 1, joined 1) with the answer
    # of their solo run
    gp, eg, hub = graph_with_tail(O, T, tail)
    late = [int(x) for x in O.sources(gp, 40)][:4]
    try:
        with T.Server(eg, group_min=1, max_batch_iters=1, join_window=0xFFFFFFFF,
                      timeout_ms=20000) as sv:
            first = sv.submit(algo, hub)
            time.sleep(0.002)
            tickets = []
            for s in late:
                tickets.append((sv.submit(algo, s), s))
                time.sleep(0.0003)
            vals, st = sv.wait(first)
            assert st["grouped"] == 1 and st["joined"] == 0
            assert np.array_equal(vals, want(O, gp, algo, hub))
            joined = 0
            for t, s in tickets:
                vals, st = sv.wait(t)
                w = want(O, gp, algo, s)
                assert np.array_equal(vals, w), (algo, s)
                assert st["checksum"] == T.values_checksum(w)
                assert st["grouped"] == 1
                joined += st["joined"]
            assert joined >= 1, "no query joined the running group"
    finally:
        eg.close()


def test_arrivals_after_the_join_window_start_a_second_group(T, O):
    # default join window (2 iterations), two groups per algorithm: a query
    # arriving after the window starts a second group at once, which shares
    # the device with the first by turns, instead of waiting for the first
    # group to drain
    gp, eg, hub = graph_with_tail(O, T, 6000)
    late = [int(x) for x in O.sources(gp, 40)][:4]
    try:
        with T.Server(eg, group_min=1, max_batch_iters=1, groups_per_algo=2,
                      timeout_ms=20000) as sv:
            first = sv.submit("sssp", hub)
            time.sleep(0.005)
            tickets = [(sv.submit("sssp", s), s) for s in late]
            vals, st0 = sv.wait(first)
            assert np.array_equal(vals, O.sssp(gp, hub))
            for j, (t, s) in enumerate(tickets):
                vals, st = sv.wait(t)
                assert np.array_equal(vals, O.sssp(gp, s)), s
                assert st["grouped"] == 1
                if j == 0:
                    assert st["queue_ms"] < st0["run_ms"] / 2, (st, st0)
    finally:
        eg.close()


@pytest.mark.parametrize("groups", [1, 2])
def test_one_or_two_groups_per_algorithm_agree(T, O, g14w, eg, groups):
    src = O.sources(g14w, 90).tolist()
    algos = ["sssp" if i % 4 == 0 else "bfs" for i in range(len(src))]
    with T.Server(eg, groups_per_algo=groups, timeout_ms=20000) as sv:
        tickets = []
        for i, (a, s) in enumerate(zip(algos, src)):
            tickets.append(sv.submit(a, s, want_values=False))
            if i % 8 == 0:
                time.sleep(0.001)
        for t, a, s in zip(tickets, algos, src):
            _, st = sv.wait(t)
            assert st["checksum"] == T.values_checksum(want(O, g14w, a, s)), (a, s)


def test_joined_sources_reuse_freed_bits(T, O):
    # a long stream through one live group: more queries than mask bits, so
    # bits of finished sources are reset and reused by later arrivals
    gp, eg, hub = graph_with_tail(O, T, 120)
    src = [int(x) for x in O.sources(gp, 150)]
    try:
        with T.Server(eg, group_min=1, join_window=0xFFFFFFFF, timeout_ms=20000) as sv:
            tickets = []
            for i, s in enumerate(src):
                tickets.append((sv.submit("bfs" if i % 3 else "sssp", s, want_values=(i % 7 == 0)), s, i))
                if i % 10 == 0:
                    time.sleep(0.001)
            joined = 0
            for t, s, i in tickets:
                vals, st = sv.wait(t)
                w = want(O, gp, "bfs" if i % 3 else "sssp", s)
                assert st["checksum"] == T.values_checksum(w), (i, s)
                if i % 7 == 0:
                    assert np.array_equal(vals, w), (i, s)
                joined += st["joined"]
            assert joined > 0
    finally:
        eg.close()


def test_group_deeper_than_the_level_bytes_falls_back_to_lone_runs(T, O):
    # BFS levels past the u8 range: the group's queries run alone instead
    gp, eg, hub = graph_with_tail(O, T, 300)
    try:
        with T.Server(eg, group_min=1, timeout_ms=20000) as sv:
            vals, st = sv.wait(sv.submit("bfs", hub))
            assert np.array_equal(vals, O.bfs(gp, hub))
            assert st["grouped"] == 2
    finally:
        eg.close()
