"""Failure paths, made on purpose without a GPU fault: a bounded device wait
that runs out (a barrier one block never reaches), and host allocations that
fail on demand.  Each returns a status and leaves the library usable."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g14(O):
    return O.rmat(14, 16)


def test_bounded_wait_reports_timeout_and_context_survives(T, O, g14):
    lib = T.load_library()
    t0 = time.perf_counter()
    st = lib.thv_debug_wait_timeout(0, 200)
    dt = time.perf_counter() - t0
    assert st == T.THV_ETIMEOUT
    assert b"exceeded 200 ms" in lib.thv_last_error()
    assert 0.15 < dt < 5.0
    # the device still runs traversals correctly
    src = int(O.sources(g14, 1)[0])
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        g.plan(int(0.4 * g.ne * 4), block_bytes=64 << 10)
        got, _ = g.run("bfs", source=src, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(g14, src))
    assert lib.thv_debug_wait_timeout(0, 0) == T.THV_EINVAL


@pytest.mark.parametrize("nth", [1, 2, 3, 4, 5, 6, 8])
def test_failed_allocations_leave_the_graph_usable(T, O, g14, nth):
    lib = T.load_library()
    src = int(O.sources(g14, 1)[0])
    with T.Graph.from_arrays(g14.off, g14.adj, "csr") as g:
        lib.thv_debug_fail_alloc_after(nth)
        failed = False
        try:
            g.plan(int(0.4 * g.ne * 4), block_bytes=64 << 10)
            g.run("bfs", source=src, timeout_ms=20000)
            g.batch_run("bfs", [src], timeout_ms=20000)
        except T.ThvError as e:
            failed = True
            assert e.status == T.THV_ENOMEM
        finally:
            lib.thv_debug_fail_alloc_after(0)
        assert failed
        g.plan(int(0.4 * g.ne * 4), block_bytes=64 << 10)
        got, _ = g.run("bfs", source=src, timeout_ms=20000)
        assert np.array_equal(got, O.bfs(g14, src))
        rows, _, _ = g.batch_run("bfs", [src], timeout_ms=20000)
        assert np.array_equal(rows[0], O.bfs(g14, src))
