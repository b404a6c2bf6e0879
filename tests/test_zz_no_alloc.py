"""The allocation-free BFS entry point (thv_bfs_noalloc) against thv_run.

thv_bfs_noalloc serves callers that cannot allocate device memory on the
call path -- a host framework that owns all device memory through its own
pool, or a latency-critical path that cannot take cudaMalloc's implicit
device synchronisation.  It keeps its scratch in a static device array
shared by every call, so this test makes two calls in a row (different
sources, then the first again) and checks each against the ordinary entry
point bit for bit: a call must not see the previous call's scratch.  The
file sorts last so a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def noalloc_bfs(lib, d_off, d_adj, nv, ne, src, d_out, stream=None):
    it = ctypes.c_uint64()
    st = lib.thv_bfs_noalloc(ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_adj.data_ptr()),
                             nv, ne, src, ctypes.c_void_p(d_out.data_ptr()),
                             None if stream is None else ctypes.c_void_p(stream.cuda_stream),
                             ctypes.byref(it))
    return st, it.value


def test_no_alloc_bfs_matches_thv_run_twice(T, O):
    import torch

    lib = T.load_library()
    g = O.rmat(16, 16)
    srcs = [int(s) for s in O.sources(g, 2)]
    with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
        eg.plan()
        want = {s: eg.run("bfs", source=s)[0] for s in srcs}
    dev = torch.device("cuda:0")
    d_off = torch.from_numpy(g.off.view(np.int64)).to(dev)
    d_adj = torch.from_numpy(g.adj.view(np.int32)).to(dev)
    d_out = torch.empty(g.nv, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    for s in srcs + [srcs[0]]:
        st, iters = noalloc_bfs(lib, d_off, d_adj, g.nv, g.ne, s, d_out)
        assert st == 0, lib.thv_last_error().decode()
        got = d_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want[s]), f"source {s}"
        assert iters > 0


def test_no_alloc_rejects_graphs_beyond_its_scratch(T):
    import torch

    lib = T.load_library()
    dev = torch.device("cuda:0")
    nv = 8 << 20  # 8 M vertices need ~134 MB of queue scratch: over 64 MiB
    d_off = torch.zeros(nv + 1, dtype=torch.int64, device=dev)
    d_adj = torch.zeros(32, dtype=torch.int32, device=dev)
    d_out = torch.empty(nv, dtype=torch.int32, device=dev)
    st, _ = noalloc_bfs(lib, d_off, d_adj, nv, 0, 0, d_out)
    assert st == T.THV_ENOMEM
    assert b"scratch" in lib.thv_last_error()


def test_no_alloc_scratch_is_clean_across_graph_sizes_and_streams(T, O):
    # a smaller graph after a larger one (fewer bitmap words, smaller
    # queues) and a larger one after it, on the default stream and on a
    # stream of the caller's: every call equals thv_run bit for bit
    import torch

    lib = T.load_library()
    dev = torch.device("cuda:0")
    side = torch.cuda.Stream(device=dev)
    cases = []
    for scale in (16, 12):
        g = O.rmat(scale, 16)
        s = int(O.sources(g, 1)[0])
        with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
            eg.plan()
            want = eg.run("bfs", source=s)[0]
        cases.append((g, s, want, torch.from_numpy(g.off.view(np.int64)).to(dev),
                      torch.from_numpy(g.adj.view(np.int32)).to(dev)))
    torch.cuda.synchronize()
    for i, (g, s, want, d_off, d_adj) in enumerate([cases[0], cases[1], cases[0]]):
        stream = side if i == 1 else None
        with torch.cuda.stream(side if stream is not None else torch.cuda.current_stream()):
            d_out = torch.full((g.nv,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        st, _ = noalloc_bfs(lib, d_off, d_adj, g.nv, g.ne, s, d_out, stream)
        assert st == 0, lib.thv_last_error().decode()
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want), f"call {i}"
