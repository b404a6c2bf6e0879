"""Config 2 at its full size against the CPU oracle, in the test suite.

RMAT scale 24 (16.8 M vertices), edge factor 16, seeded as the benchmark
generates it; HBM budget 40% of the format's edge bytes, the rest read
zero-copy from pinned host memory:
- SSSP on the WCSR graph (weights 1..64, packed into 4-byte edges) from
  three sources, every distance against the OpenMP oracle (label-correcting
  to the same fixed point as Dijkstra);
- CC by min-label propagation on the symmetrised CSR graph, every label
  against the oracle.
The reference loops these replace: src/sssp/sssp.cu:10-570 and
src/cc/cc.cu:71-614.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x54484592  # the benchmark's generator seed


def oracle_of(O, g, algo, src=0):
    off, edges, _ = g.host_arrays()
    out = np.empty(g.nv, np.uint32)
    L = O.lib()
    if algo == "sssp":
        rc = L.thvo_sssp_par(g.nv, off.ctypes.data, edges.ctypes.data, None, 2, src, out.ctypes.data)
    else:
        rc = L.thvo_cc_par(g.nv, off.ctypes.data, edges.ctypes.data, 1, out.ctypes.data)
    assert rc == 0
    return out


def test_sssp_rmat24_wcsr_hbm40(T, O):
    with T.Graph.generate_rmat(24, 16, seed=SEED, fmt="wcsr") as g:
        info = g.plan(int(0.4 * g.ne * g.esz))
        assert info["host_edge_bytes"] > 0 and info["resident_edge_bytes"] > 0
        for src in (1, 7, 1000):
            got, st = g.run("sssp", source=src)
            assert st["link_edge_bytes"] > 0
            assert np.array_equal(got, oracle_of(O, g, "sssp", src)), src


def test_cc_label_propagation_rmat24_sym_hbm40(T, O):
    with T.Graph.generate_rmat(24, 16, seed=SEED, symmetric=True, fmt="csr") as g:
        g.plan(int(0.4 * g.ne * g.esz))
        got, st = g.run("cc", label_propagation=True)
        assert st["link_edge_bytes"] > 0
        assert np.array_equal(got, oracle_of(O, g, "cc"))
