"""CPU oracle bindings (TEST INFRASTRUCTURE ONLY).

The checker for the GPU engine: ctypes bindings to ``oracle/libthv_oracle.so``
(plain C + OpenMP, oracle/thv_oracle.c).  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference arm may import this module; the
engine (thievory_b200) never does.

Semantics follow the reference's value encoding (src/graph.cuh:244-265): BFS
and SSSP store distance + 1 with the source at 1 and unreached vertices at
n + 1; CC labels are the minimum id of any vertex that reaches the vertex.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libthv_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
SEED = 0x54484592  # "THEV" + 60: vertex 1 is non-isolated at scales 20, 24 and 26

_lib = None


def build() -> None:
    subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        P, U32, U64, D, I = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_int
        sig = {
            "thvo_mix64": ([U64], U64),
            "thvo_permute": ([U64, U32, U64], U64),
            "thvo_weight": ([U64, U32, U32], U32),
            "thvo_rmat_thresholds": ([D, D, D, P], None),
            "thvo_rmat_edges": ([U32, U64, P, U64, U64, P, P], None),
            "thvo_build_csr": ([U64, U64, P, P, I, P, ctypes.POINTER(ctypes.c_void_p),
                                ctypes.POINTER(ctypes.c_uint64)], I),
            "thvo_generate": ([U32, U32, U64, D, D, D, I, P, ctypes.POINTER(ctypes.c_void_p),
                               ctypes.POINTER(ctypes.c_uint64)], I),
            "thvo_weights": ([U64, P, P, U64, P], None),
            "thvo_transpose": ([U64, U64, P, P, P, P, P], None),
            "thvo_sources": ([U64, P, U64, U32, P], I),
            "thvo_bfs": ([U64, P, P, U32, U32, P], I),
            "thvo_bfs_par": ([U64, P, P, U32, U32, P], I),
            "thvo_cc": ([U64, P, P, U32, P], I),
            "thvo_cc_par": ([U64, P, P, U32, P], I),
            "thvo_sssp": ([U64, P, P, P, U32, U32, P], I),
            "thvo_sssp_par": ([U64, P, P, P, U32, U32, P], I),
            "thvo_pagerank": ([U64, P, P, U32, U32, D, P], I),
            "thvo_pagerank_csc": ([U64, P, P, P, U32, D, P], I),
            "thvo_pagerank_ref_pull": ([U64, P, P, P, U32, P, P], I),
            "thvo_pagerank_ref_push": ([U64, P, P, U32, U32, P, P], I),
            "thvo_reached_edges": ([U64, P, P], U64),
            "thvo_write_csr": ([ctypes.c_char_p, U64, U64, P, P, P], I),
            "thvo_write_csc": ([ctypes.c_char_p, U64, U64, P, P, P], I),
            "thvo_write_wcsr": ([ctypes.c_char_p, U64, U64, P, P, P], I),
            "thvo_write_values": ([ctypes.c_char_p, P, U64, U32], I),
            "thvo_now": ([], D),
            "thvo_threads": ([], I),
            "thvo_set_threads": ([I], None),
        }
        for n, (a, r) in sig.items():
            f = getattr(L, n)
            f.argtypes = a
            f.restype = r
        L.free = ctypes.CDLL(None).free
        L.free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class CSR:
    """Host CSR: off (nv+1 u64), adj (ne u32), optional w (ne u32)."""

    def __init__(self, off, adj, w=None):
        self.off = _c(off, np.uint64)
        self.adj = _c(adj, np.uint32)
        self.w = None if w is None else _c(w, np.uint32)

    @property
    def nv(self):
        return len(self.off) - 1

    @property
    def ne(self):
        return int(self.off[-1])

    def wcsr_edges(self) -> np.ndarray:
        """Interleaved {dst, w} (ne, 2) array (the .wcsr edge layout)."""
        w = self.w if self.w is not None else np.full(self.ne, 20, np.uint32)
        return np.ascontiguousarray(np.stack([self.adj, w], axis=1))


def from_edges(nv: int, src, dst, symmetric: bool = False) -> CSR:
    """Dedup, drop self-loops, sort by (src,dst)."""
    L = lib()
    s, d = _c(src, np.uint32), _c(dst, np.uint32)
    off = np.zeros(nv + 1, np.uint64)
    pa, ne = ctypes.c_void_p(), ctypes.c_uint64()
    if L.thvo_build_csr(nv, len(s), _p(s), _p(d), int(symmetric), _p(off), ctypes.byref(pa),
                        ctypes.byref(ne)) != 0:
        raise MemoryError("thvo_build_csr")
    adj = np.ctypeslib.as_array((ctypes.c_uint32 * max(ne.value, 1)).from_address(pa.value))[: ne.value].copy()
    L.free(pa)
    return CSR(off, adj)


def rmat(scale: int, edge_factor: int = 16, seed: int = SEED, a=0.57, b=0.19, c=0.19,
         symmetric: bool = False, weighted: bool = False) -> CSR:
    L = lib()
    nv = 1 << scale
    off = np.zeros(nv + 1, np.uint64)
    pa, ne = ctypes.c_void_p(), ctypes.c_uint64()
    if L.thvo_generate(scale, edge_factor, seed, a, b, c, int(symmetric), _p(off),
                       ctypes.byref(pa), ctypes.byref(ne)) != 0:
        raise MemoryError("thvo_generate")
    n = ne.value
    adj = np.ctypeslib.as_array((ctypes.c_uint32 * max(n, 1)).from_address(pa.value))[:n].copy()
    L.free(pa)
    g = CSR(off, adj)
    if weighted:
        g.w = weights(g, seed)
    return g


def rmat_raw(scale: int, count: int, seed: int = SEED, a=0.57, b=0.19, c=0.19, first: int = 0):
    L = lib()
    thr = np.zeros(3, np.uint32)
    L.thvo_rmat_thresholds(a, b, c, _p(thr))
    s = np.empty(count, np.uint32)
    d = np.empty(count, np.uint32)
    L.thvo_rmat_edges(scale, seed, _p(thr), first, count, _p(s), _p(d))
    return s, d


def weights(g: CSR, seed: int = SEED) -> np.ndarray:
    w = np.empty(g.ne, np.uint32)
    lib().thvo_weights(g.nv, _p(g.off), _p(g.adj), seed, _p(w))
    return w


def transpose(g: CSR):
    """CSR -> (in_off, in_adj sorted by (dst,src), outdeg)."""
    in_off = np.zeros(g.nv + 1, np.uint64)
    in_adj = np.empty(max(g.ne, 1), np.uint32)
    outdeg = np.empty(g.nv, np.uint32)
    lib().thvo_transpose(g.nv, g.ne, _p(g.off), _p(g.adj), _p(in_off), _p(in_adj), _p(outdeg))
    return in_off, in_adj[: g.ne], outdeg


def sources(g: CSR, n: int, seed: int = SEED) -> np.ndarray:
    out = np.empty(n, np.uint32)
    if lib().thvo_sources(g.nv, _p(g.off), seed, n, _p(out)) != 0:
        raise ValueError("no vertex with out-degree > 0")
    return out


def _adj_stride(g: CSR, interleaved: bool):
    if interleaved:
        return g.wcsr_edges(), 2
    return g.adj, 1


def bfs(g: CSR, src: int, parallel: bool = False) -> np.ndarray:
    out = np.empty(g.nv, np.uint32)
    f = lib().thvo_bfs_par if parallel else lib().thvo_bfs
    if f(g.nv, _p(g.off), _p(g.adj), 1, src, _p(out)) != 0:
        raise ValueError("bfs: bad source")
    return out


def cc(g: CSR, parallel: bool = False) -> np.ndarray:
    out = np.empty(g.nv, np.uint32)
    f = lib().thvo_cc_par if parallel else lib().thvo_cc
    if f(g.nv, _p(g.off), _p(g.adj), 1, _p(out)) != 0:
        raise MemoryError("cc")
    return out


def sssp(g: CSR, src: int, parallel: bool = False) -> np.ndarray:
    if g.w is None:
        raise ValueError("sssp needs weights")
    out = np.empty(g.nv, np.uint32)
    f = lib().thvo_sssp_par if parallel else lib().thvo_sssp
    if f(g.nv, _p(g.off), _p(g.adj), _p(g.w), 1, src, _p(out)) != 0:
        raise ValueError("sssp: bad source")
    return out


def pagerank(g: CSR, iters: int = 20, damping: float = 0.85) -> np.ndarray:
    out = np.empty(g.nv, np.float64)
    if lib().thvo_pagerank(g.nv, _p(g.off), _p(g.adj), 1, iters, damping, _p(out)) != 0:
        raise MemoryError("pagerank")
    return out


def pagerank_csc(in_off, in_adj, outdeg, iters: int = 20, damping: float = 0.85) -> np.ndarray:
    in_off, in_adj, outdeg = _c(in_off, np.uint64), _c(in_adj, np.uint32), _c(outdeg, np.uint32)
    nv = len(in_off) - 1
    out = np.empty(nv, np.float64)
    if lib().thvo_pagerank_csc(nv, _p(in_off), _p(in_adj), _p(outdeg), iters, damping, _p(out)) != 0:
        raise MemoryError("pagerank_csc")
    return out


def pagerank_ref_pull(in_off, in_adj, outdeg, max_rounds: int = 100000):
    """The reference engine's pull PageRank (FP64, tolerance-driven) over a
    CSC; returns (values, rounds)."""
    nv = len(in_off) - 1
    io, ia, od = _c(in_off, np.uint64), _c(in_adj, np.uint32), _c(outdeg, np.uint32)
    out = np.empty(nv, np.float64)
    rounds = np.zeros(1, np.uint32)
    rc = lib().thvo_pagerank_ref_pull(nv, _p(io), _p(ia), _p(od), max_rounds, _p(out), _p(rounds))
    if rc != 0:
        raise RuntimeError(f"pagerank_ref_pull: {rc}")
    return out, int(rounds[0])


def pagerank_ref_push(g: CSR, max_rounds: int = 100000):
    """The reference engine's push PageRank (FP64 residual form,
    tolerance-driven) over the out-edges; returns (values, rounds)."""
    out = np.empty(g.nv, np.float64)
    rounds = np.zeros(1, np.uint32)
    rc = lib().thvo_pagerank_ref_push(g.nv, _p(g.off), _p(g.adj), 1, max_rounds, _p(out),
                                      _p(rounds))
    if rc != 0:
        raise RuntimeError(f"pagerank_ref_push: {rc}")
    return out, int(rounds[0])


def reached_edges(g: CSR, values: np.ndarray) -> int:
    v = _c(values, np.uint32)
    return int(lib().thvo_reached_edges(g.nv, _p(g.off), _p(v)))


def write_csr(path: str, g: CSR) -> None:
    if lib().thvo_write_csr(path.encode(), g.nv, g.ne, _p(g.off), _p(g.adj), _p(g.w)) != 0:
        raise OSError(path)


def write_wcsr(path: str, g: CSR) -> None:
    if lib().thvo_write_wcsr(path.encode(), g.nv, g.ne, _p(g.off), _p(g.adj), _p(g.w)) != 0:
        raise OSError(path)


def write_csc(path: str, g: CSR) -> None:
    in_off, in_adj, outdeg = transpose(g)
    if lib().thvo_write_csc(path.encode(), g.nv, g.ne, _p(in_off), _p(in_adj), _p(outdeg)) != 0:
        raise OSError(path)


def threads() -> int:
    return int(lib().thvo_threads())


def set_threads(n: int) -> None:
    """OpenMP threads of later oracle calls (a launcher may have set 1)."""
    lib().thvo_set_threads(int(n))
