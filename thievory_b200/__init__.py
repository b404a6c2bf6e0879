"""thievory_b200 -- B200-native out-of-memory graph engine (host-side mirror).

This module binds the engine's C ABI (``include/thv.h``, built into
``thievory_b200/libthv.so``) with ctypes and mirrors the reference's
operator interface:

* ``BFS32 / CC32 / SSSP32 / PR32 / PR32_PUSH`` keep the reference driver
  names and argument meaning (src/bfs/bfs.cuh:8, src/cc/cc.cuh:8,
  src/sssp/sssp.cuh:8, src/pr/pr.cuh:8-14): load a graph file, run it
  ``n_runs`` times, print "Average execution time", dump
  ``results/values.bin``.  Where the reference calls ``exit()``
  (src/common.cuh:51-62, src/graph.cuh:702-705) these raise ``ThvError``.
* ``Graph`` is the object API used by tests and bench.py.

The CUDA library is required: importing works without a GPU (to inspect the
ABI), but every call that computes fails loudly when the library or a GPU is
missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import time
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libthv.so")

# status codes (include/thv.h)
THV_OK, THV_EINVAL, THV_EIO, THV_EFORMAT, THV_ENOMEM, THV_ECUDA = 0, 1, 2, 3, 4, 5
THV_ETIMEOUT, THV_EUNSUPPORTED, THV_EBUSY, THV_ENOTREADY, THV_EDEVICE = 6, 7, 8, 9, 10

FMT = {"csr": 0, "csc": 1, "wcsr": 2}
ALGO = {"bfs": 0, "cc": 1, "sssp": 2, "pr_push": 3, "pr_pull": 4}
PLACE = {"densest": 0, "prefix": 1, "access": 2}
OPEN_WEIGHTS = 1


class ThvError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: status {status}: {message}")


class _RunOpts(ctypes.Structure):
    _fields_ = [("source", ctypes.c_uint32), ("pr_iters", ctypes.c_uint32),
                ("pr_damping", ctypes.c_double), ("sssp_delta", ctypes.c_uint32),
                ("timeout_ms", ctypes.c_uint32), ("stream", ctypes.c_void_p),
                ("small_degree", ctypes.c_uint32), ("chunk_edges", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("sssp_growth", ctypes.c_uint32)]


class _Stats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
                ("iterations", ctypes.c_uint64), ("edges_expanded", ctypes.c_uint64),
                ("hbm_edge_bytes", ctypes.c_uint64), ("link_edge_bytes", ctypes.c_uint64),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint32), ("bottom_up_levels", ctypes.c_uint32),
                ("checksum", ctypes.c_uint64)]

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class _PlanOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("block_bytes", ctypes.c_uint64),
                ("policy", ctypes.c_uint32), ("small_list_degree", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class _PlanInfo(ctypes.Structure):
    _fields_ = [("num_blocks", ctypes.c_uint64), ("resident_blocks", ctypes.c_uint64),
                ("resident_edge_bytes", ctypes.c_uint64), ("host_edge_bytes", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64), ("small_list_degree", ctypes.c_uint64),
                ("small_list_bytes", ctypes.c_uint64), ("small_list_vertices", ctypes.c_uint64)]


class _GraphInfo(ctypes.Structure):
    _fields_ = [("nv", ctypes.c_uint64), ("ne", ctypes.c_uint64), ("fmt", ctypes.c_uint32),
                ("esz", ctypes.c_uint32), ("device", ctypes.c_uint32),
                ("weighted", ctypes.c_uint32), ("mem_esz", ctypes.c_uint32),
                ("weight_bits", ctypes.c_uint32), ("sorted", ctypes.c_uint32),
                ("symmetric", ctypes.c_uint32)]


class _RmatOpts(ctypes.Structure):
    _fields_ = [("scale", ctypes.c_uint32), ("edge_factor", ctypes.c_uint32),
                ("seed", ctypes.c_uint64), ("a", ctypes.c_double), ("b", ctypes.c_double),
                ("c", ctypes.c_double), ("symmetric", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class _BatchOpts(ctypes.Structure):
    _fields_ = [("group", ctypes.c_uint32), ("timeout_ms", ctypes.c_uint32),
                ("stream", ctypes.c_void_p), ("small_degree", ctypes.c_uint32),
                ("chunk_edges", ctypes.c_uint32), ("sssp_delta", ctypes.c_uint32),
                ("tune", ctypes.c_uint32), ("sssp_growth", ctypes.c_uint32),
                ("mid_degree", ctypes.c_uint32), ("small_group", ctypes.c_uint32),
                ("mid_group", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


class _BatchConfig(ctypes.Structure):
    _fields_ = [("small_degree", ctypes.c_uint32), ("mid_degree", ctypes.c_uint32),
                ("chunk_edges", ctypes.c_uint32), ("threads", ctypes.c_uint32),
                ("small_group", ctypes.c_uint32), ("mid_group", ctypes.c_uint32),
                ("tuned", ctypes.c_uint32), ("pad", ctypes.c_uint32)]

    def to_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "pad"}


class _ServeOpts(ctypes.Structure):
    _fields_ = [("max_slots", ctypes.c_uint32), ("queue_capacity", ctypes.c_uint32),
                ("mem_budget_bytes", ctypes.c_uint64), ("timeout_ms", ctypes.c_uint32),
                ("max_batch_iters", ctypes.c_uint32), ("group_min", ctypes.c_uint32),
                ("replan_every", ctypes.c_uint32), ("join_window", ctypes.c_uint32),
                ("groups_per_algo", ctypes.c_uint32)]


class _QueryStats(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("checksum", ctypes.c_uint64),
                ("iterations", ctypes.c_uint32), ("slot", ctypes.c_uint32),
                ("status", ctypes.c_int32), ("grouped", ctypes.c_uint32),
                ("joined", ctypes.c_uint32), ("pad", ctypes.c_uint32)]

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


# Every function include/thv.h declares (tests check the library exports them).
ABI_FUNCTIONS = [
    "thv_open", "thv_from_arrays", "thv_generate_rmat", "thv_save", "thv_close",
    "thv_info", "thv_set_edge_packing", "thv_set_symmetric", "thv_convert", "thv_host_arrays", "thv_plan", "thv_get_plan", "thv_get_blocks", "thv_get_block_access", "thv_save_plan", "thv_load_plan", "thv_run",
    "thv_values", "thv_write_values", "thv_batch_run", "thv_batch_tuned", "thv_serve_start",
    "thv_serve_submit", "thv_serve_poll", "thv_serve_wait", "thv_serve_stop",
    "thv_pick_sources", "thv_bfs_noalloc", "thv_link_bandwidth", "thv_last_error", "thv_status_str", "thv_abi_version",
    "thv_debug_fail_alloc_after", "thv_debug_wait_timeout",
]

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libthv.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"thievory_b200: CUDA library missing at {path}; "
                          "run __graft_entry__.build() (make -C thievory_b200/csrc)")
    lib = ctypes.CDLL(path)
    P, U32, U64, I32, D = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
    pp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "thv_open": ([ctypes.c_char_p, U32, U32, I32, pp], I32),
        "thv_from_arrays": ([U64, U64, P, P, U32, U32, P, I32, pp], I32),
        "thv_generate_rmat": ([ctypes.POINTER(_RmatOpts), U32, I32, pp], I32),
        "thv_save": ([P, ctypes.c_char_p], I32),
        "thv_close": ([P], I32),
        "thv_info": ([P, ctypes.POINTER(_GraphInfo)], I32),
        "thv_set_edge_packing": ([P, I32], I32),
        "thv_set_symmetric": ([P, I32], I32),
        "thv_convert": ([ctypes.c_char_p, ctypes.c_char_p, U32, U32, U32, I32,
                         ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)], I32),
        "thv_host_arrays": ([P, pp, pp, pp], I32),
        "thv_plan": ([P, ctypes.POINTER(_PlanOpts)], I32),
        "thv_get_plan": ([P, ctypes.POINTER(_PlanInfo)], I32),
        "thv_get_blocks": ([P, U64, P, P, ctypes.POINTER(ctypes.c_uint64)], I32),
        "thv_get_block_access": ([P, U64, P, ctypes.POINTER(ctypes.c_uint64)], I32),
        "thv_save_plan": ([P, ctypes.c_char_p], I32),
        "thv_load_plan": ([P, ctypes.c_char_p], I32),
        "thv_link_bandwidth": ([I32, U64, ctypes.POINTER(D), ctypes.POINTER(D)], I32),
        "thv_pick_sources": ([P, U64, U32, P], I32),
        "thv_bfs_noalloc": ([P, P, U64, U64, U32, P, P, ctypes.POINTER(ctypes.c_uint64)], I32),
        "thv_run": ([P, U32, ctypes.POINTER(_RunOpts), P, ctypes.POINTER(_Stats)], I32),
        "thv_values": ([P, P], I32),
        "thv_write_values": ([ctypes.c_char_p, P, U64, U32], I32),
        "thv_batch_run": ([P, U32, P, U32, ctypes.POINTER(_BatchOpts), P, P,
                           ctypes.POINTER(_Stats)], I32),
        "thv_batch_tuned": ([P, U32, ctypes.POINTER(_BatchConfig)], I32),
        "thv_serve_start": ([P, ctypes.POINTER(_ServeOpts), pp], I32),
        "thv_serve_submit": ([P, U32, U32, P, ctypes.POINTER(ctypes.c_uint64)], I32),
        "thv_serve_poll": ([P, U64, ctypes.POINTER(_QueryStats)], I32),
        "thv_serve_wait": ([P, U64, ctypes.POINTER(_QueryStats), U32], I32),
        "thv_serve_stop": ([P], I32),
        "thv_last_error": ([], ctypes.c_char_p),
        "thv_status_str": ([I32], ctypes.c_char_p),
        "thv_abi_version": ([], U32),
        "thv_debug_fail_alloc_after": ([U32], None),
        "thv_debug_wait_timeout": ([I32, U32], I32),
    }
    for name, (argt, rest) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = rest
    _lib = lib
    return lib


def _check(status: int, where: str) -> None:
    if status != THV_OK:
        lib = load_library()
        raise ThvError(status, where, lib.thv_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def value_dtype(algo: str):
    return np.float64 if algo.startswith("pr") else np.uint32


def convert(txt_path: str, out_path: str, fmt: str = "csr", skip: int = 4,
            weighted: bool = False, undirected: bool = False, device: int = 0):
    """Text edge list -> .csr/.csc/.wcsr with the reference converter's bytes
    (converter/converter.cpp); sorts on the GPU.  Returns (nv, ne)."""
    nv, ne = ctypes.c_uint64(), ctypes.c_uint64()
    flags = (1 if weighted else 0) | (2 if undirected else 0)
    _check(load_library().thv_convert(txt_path.encode(), out_path.encode(), FMT[fmt], skip, flags,
                                      device, ctypes.byref(nv), ctypes.byref(ne)), "thv_convert")
    return int(nv.value), int(ne.value)


class Graph:
    """A graph held by the engine: pinned host edges plus device state."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle
        self._refresh()

    def _refresh(self) -> None:
        info = _GraphInfo()
        _check(load_library().thv_info(self._h, ctypes.byref(info)), "thv_info")
        self.nv, self.ne = int(info.nv), int(info.ne)
        self.fmt = {v: k for k, v in FMT.items()}[info.fmt]
        # esz: the format's bytes per edge; mem_esz: as stored (4 when packed)
        self.esz, self.weighted, self.device = int(info.esz), bool(info.weighted), int(info.device)
        self.mem_esz, self.weight_bits = int(info.mem_esz), int(info.weight_bits)
        self.sorted, self.symmetric = bool(info.sorted), bool(info.symmetric)

    def set_symmetric(self, symmetric: bool = True) -> None:
        """Assert that every edge has its reverse: CC then runs as sampling
        union-find and skips most adjacency lists."""
        _check(load_library().thv_set_symmetric(self._h, 1 if symmetric else 0), "thv_set_symmetric")
        self._refresh()

    def set_edge_packing(self, packed: bool) -> None:
        """Store weighted edges packed in 4 bytes (default) or as {dst, w}
        pairs; drops the plan.  Host views from host_arrays() are invalid
        afterwards."""
        _check(load_library().thv_set_edge_packing(self._h, 1 if packed else 0),
               "thv_set_edge_packing")
        self._refresh()

    # -- construction -------------------------------------------------------
    @classmethod
    def open(cls, path: str, fmt: str = "csr", weights: bool = False, device: int = 0) -> "Graph":
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.thv_open(path.encode(), FMT[fmt], OPEN_WEIGHTS if weights else 0, device,
                            ctypes.byref(h)), "thv_open")
        return cls(h)

    @classmethod
    def from_arrays(cls, off: np.ndarray, edges: np.ndarray, fmt: str = "csr",
                    outdeg: Optional[np.ndarray] = None, device: int = 0) -> "Graph":
        lib = load_library()
        off = np.ascontiguousarray(off, dtype=np.uint64)
        edges = np.ascontiguousarray(edges, dtype=np.uint32)
        nv = len(off) - 1
        esz = 8 if (edges.ndim == 2 and edges.shape[1] == 2) else 4
        ne = edges.shape[0] if edges.ndim == 2 else edges.size
        od = None if outdeg is None else np.ascontiguousarray(outdeg, dtype=np.uint32)
        h = ctypes.c_void_p()
        _check(lib.thv_from_arrays(nv, ne, _ptr(off), _ptr(edges), esz, FMT[fmt],
                                   None if od is None else _ptr(od), device, ctypes.byref(h)),
               "thv_from_arrays")
        return cls(h)

    @classmethod
    def generate_rmat(cls, scale: int, edge_factor: int = 16, seed: int = 0x54484592,
                      a: float = 0.57, b: float = 0.19, c: float = 0.19,
                      symmetric: bool = False, fmt: str = "csr", device: int = 0) -> "Graph":
        lib = load_library()
        o = _RmatOpts(scale, edge_factor, seed, a, b, c, 1 if symmetric else 0, 0)
        h = ctypes.c_void_p()
        _check(lib.thv_generate_rmat(ctypes.byref(o), FMT[fmt], device, ctypes.byref(h)),
               "thv_generate_rmat")
        return cls(h)

    # -- plan ---------------------------------------------------------------
    def plan(self, hbm_budget_bytes: Optional[int] = None, block_bytes: int = 0,
             policy: str = "densest", small_list_degree: int = 0,
             track_access: bool = False) -> dict:
        """Choose the HBM-resident edges.  small_list_degree: lists shorter
        than this in host blocks are cached in HBM first (0 = default: 64
        for CSR/WCSR, off for CSC; 1 = off; PageRank ignores the cache).
        policy "access" keeps the blocks that read the most link bytes
        under earlier plans made with track_access."""
        lib = load_library()
        o = _PlanOpts(2**64 - 1 if hbm_budget_bytes is None else int(hbm_budget_bytes),
                      int(block_bytes), PLACE[policy], int(small_list_degree),
                      1 if track_access else 0, 0)
        _check(lib.thv_plan(self._h, ctypes.byref(o)), "thv_plan")
        return self.plan_info()

    def plan_info(self) -> dict:
        pi = _PlanInfo()
        _check(load_library().thv_get_plan(self._h, ctypes.byref(pi)), "thv_get_plan")
        return {k: int(getattr(pi, k)) for k, _ in pi._fields_}

    def block_access(self) -> np.ndarray:
        """Adjacency bytes read from each block (HBM or link) under the
        current tracked plan."""
        lib = load_library()
        nb = ctypes.c_uint64()
        _check(lib.thv_get_block_access(self._h, 0, None, ctypes.byref(nb)), "thv_get_block_access")
        out = np.zeros(nb.value, np.uint64)
        _check(lib.thv_get_block_access(self._h, nb.value, _ptr(out), ctypes.byref(nb)),
               "thv_get_block_access")
        return out

    def save_plan(self, path: str) -> None:
        _check(load_library().thv_save_plan(self._h, path.encode()), "thv_save_plan")

    def load_plan(self, path: str) -> dict:
        _check(load_library().thv_load_plan(self._h, path.encode()), "thv_load_plan")
        return self.plan_info()

    def blocks(self):
        """(vbegin[nb+1] u32, resident[nb] bool) of the current plan."""
        lib = load_library()
        nb = ctypes.c_uint64()
        _check(lib.thv_get_blocks(self._h, 0, None, None, ctypes.byref(nb)), "thv_get_blocks")
        vb = np.empty(nb.value + 1, np.uint32)
        res = np.empty(max(nb.value, 1), np.uint8)
        _check(lib.thv_get_blocks(self._h, nb.value, _ptr(vb), _ptr(res), ctypes.byref(nb)),
               "thv_get_blocks")
        return vb, res[: nb.value].astype(bool)

    # -- runs ---------------------------------------------------------------
    def run(self, algo: str, source: int = 1, pr_iters: int = 20, pr_damping: float = 0.85,
            out: Optional[np.ndarray] = None, want_values: bool = True, stream: int = 0,
            sssp_delta: int = 0, timeout_ms: int = 0, small_degree: int = 0,
            chunk_edges: int = 0, checksum: bool = False, compaction: str = "",
            sssp_growth: int = 0, top_down_only: bool = False, label_propagation: bool = False,
            pr_reference: bool = False, pr_max_rounds: int = 0):
        """Run algo; returns (values or None, stats dict).  compaction:
        "" (per-algorithm default), "scan" or "queue"; sssp_growth: SSSP
        window growth per advance (0 = default 32, 1 = fixed windows).
        pr_reference: PageRank with the reference engine's semantics (FP64,
        rounds until converged to 1e-3; THV_RUN_PR_REFERENCE), at most
        pr_max_rounds rounds (0 = 100000)."""
        lib = load_library()
        flags = ((1 if checksum else 0) | (2 if compaction == "scan" else 0)
                 | (4 if compaction == "queue" else 0) | (8 if top_down_only else 0)
                 | (16 if label_propagation else 0) | (32 if pr_reference else 0))
        o = _RunOpts(source, pr_max_rounds if pr_reference else pr_iters, pr_damping, sssp_delta,
                     timeout_ms,
                     ctypes.c_void_p(stream) if stream else None, small_degree, chunk_edges,
                     flags, sssp_growth)
        st = _Stats()
        buf = None
        if want_values:
            buf = out if out is not None else np.empty(self.nv, dtype=value_dtype(algo))
        _check(lib.thv_run(self._h, ALGO[algo], ctypes.byref(o),
                           None if buf is None else _ptr(buf), ctypes.byref(st)), f"thv_run({algo})")
        return buf, st.to_dict()

    def values(self, algo: str) -> np.ndarray:
        buf = np.empty(self.nv, dtype=value_dtype(algo))
        _check(load_library().thv_values(self._h, _ptr(buf)), "thv_values")
        return buf

    def batch_run(self, algo: str, sources: Sequence[int], group: int = 64,
                  want_values: bool = True, stream: int = 0, small_degree: int = 0,
                  chunk_edges: int = 0, timeout_ms: int = 0, sssp_delta: int = 0,
                  tune: bool = False, sssp_growth: int = 0, mid_degree: int = 0,
                  small_group: int = 0, mid_group: int = 0):
        """Batched BFS/SSSP; returns (values [n, nv] or None, checksums [n], stats).

        small_degree / mid_degree / chunk_edges / small_group / mid_group set
        the degree buckets of the expansion explicitly (thv_batch_opts); all
        zero takes the tuned configuration (tune=True tunes it on the first
        group when none is cached) or the default."""
        lib = load_library()
        src = np.ascontiguousarray(sources, dtype=np.uint32)
        out = np.empty((len(src), self.nv), dtype=np.uint32) if want_values else None
        sums = np.empty(len(src), dtype=np.uint64)
        o = _BatchOpts(group, timeout_ms, ctypes.c_void_p(stream) if stream else None,
                       small_degree, chunk_edges, sssp_delta, 1 if tune else 0, sssp_growth,
                       mid_degree, small_group, mid_group, 0)
        st = _Stats()
        _check(lib.thv_batch_run(self._h, ALGO[algo], _ptr(src), len(src), ctypes.byref(o),
                                 None if out is None else _ptr(out), _ptr(sums),
                                 ctypes.byref(st)), f"thv_batch_run({algo})")
        return out, sums, st.to_dict()

    def batch_tuned(self, algo: str) -> dict:
        """The batch kernel's configuration for this graph (thv_batch_tuned)."""
        c = _BatchConfig()
        _check(load_library().thv_batch_tuned(self._h, ALGO[algo], ctypes.byref(c)),
               f"thv_batch_tuned({algo})")
        return c.to_dict()

    def pick_sources(self, n: int, seed: int = 0x54484592) -> np.ndarray:
        """n seeded sources uniform over vertices with out-degree > 0."""
        out = np.empty(n, np.uint32)
        _check(load_library().thv_pick_sources(self._h, seed, n, _ptr(out)), "thv_pick_sources")
        return out

    def save(self, path: str) -> None:
        _check(load_library().thv_save(self._h, path.encode()), "thv_save")

    def host_arrays(self):
        """Zero-copy numpy views of the host CSR/CSC (valid until close)."""
        lib = load_library()
        po, pe, pd = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(lib.thv_host_arrays(self._h, ctypes.byref(po), ctypes.byref(pe), ctypes.byref(pd)),
               "thv_host_arrays")
        off = np.ctypeslib.as_array((ctypes.c_uint64 * (self.nv + 1)).from_address(po.value))
        n32 = self.ne * (self.esz // 4)
        edges = (np.ctypeslib.as_array((ctypes.c_uint32 * n32).from_address(pe.value))
                 if n32 else np.zeros(0, np.uint32))
        if self.esz == 8:
            edges = edges.reshape(-1, 2)
        outdeg = (np.ctypeslib.as_array((ctypes.c_uint32 * self.nv).from_address(pd.value))
                  if pd.value else None)
        return off, edges, outdeg

    def close(self) -> None:
        if self._h:
            load_library().thv_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching query server over a Graph (thv_serve_*).

    submit() never blocks; results land in the array given at submit time
    (kept alive here until the ticket completes)."""

    def __init__(self, graph: Graph, max_slots: int = 64, queue_capacity: int = 0,
                 mem_budget_bytes: int = 0, timeout_ms: int = 0, max_batch_iters: int = 0,
                 group_min: int = 0, replan_every: int = 0, join_window: int = 0,
                 groups_per_algo: int = 0):
        """group_min: waiting queries of one algorithm that run as a batched
        group (0 = measured defaults: BFS 4, SSSP 6; 0xFFFFFFFF = no
        batching: slot admission)."""
        lib = load_library()
        self.graph = graph
        self._bufs = {}
        o = _ServeOpts(max_slots, queue_capacity, mem_budget_bytes, timeout_ms, max_batch_iters,
                       group_min, replan_every, join_window, groups_per_algo)
        self._h = ctypes.c_void_p()
        _check(lib.thv_serve_start(graph._h, ctypes.byref(o), ctypes.byref(self._h)),
               "thv_serve_start")

    def submit(self, algo: str, source: int, want_values: bool = True) -> int:
        out = np.empty(self.graph.nv, np.uint32) if want_values else None
        t = ctypes.c_uint64()
        _check(load_library().thv_serve_submit(self._h, ALGO[algo], int(source),
                                               None if out is None else _ptr(out),
                                               ctypes.byref(t)), "thv_serve_submit")
        self._bufs[int(t.value)] = out
        return int(t.value)

    def poll(self, ticket: int):
        """None while running; else (values or None, stats dict)."""
        qs = _QueryStats()
        s = load_library().thv_serve_poll(self._h, ticket, ctypes.byref(qs))
        if s == THV_ENOTREADY:
            return None
        out = self._bufs.pop(ticket, None)
        _check(s, "thv_serve_poll")
        return out, qs.to_dict()

    def wait(self, ticket: int, timeout_ms: int = 60000):
        qs = _QueryStats()
        s = load_library().thv_serve_wait(self._h, ticket, ctypes.byref(qs), timeout_ms)
        out = self._bufs.pop(ticket, None)
        _check(s, "thv_serve_wait")
        return out, qs.to_dict()

    def stop(self) -> None:
        if self._h:
            h, self._h = self._h, None
            _check(load_library().thv_serve_stop(h), "thv_serve_stop")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()


# ---------------------------------------------------------------------------
# Reference-named drivers (src/{bfs,cc,sssp,pr}/*.cuh).  n_neighbor_gpus must
# be 0: this engine runs on one GPU.


def _driver(file_path: str, fmt: str, weights: bool, algo: str, src: int, n_runs: int,
            n_neighbor_gpus: int, hbm_budget_bytes: Optional[int], values_path: str):
    if n_neighbor_gpus != 0:
        raise ThvError(THV_EUNSUPPORTED, algo, "neighbour GPUs are not supported (use 0)")
    with Graph.open(file_path, fmt, weights=weights) as g:
        g.plan(hbm_budget_bytes)
        total = 0.0
        for _ in range(n_runs):
            _, st = g.run(algo, source=src, want_values=False)
            print(f"Execution time: : {st['wall_ms']} ms")
            total += st["wall_ms"]
        avg = total / max(n_runs, 1)
        print(f"Average execution time: {avg} ms")
        vals = g.values(algo)
        if os.path.isdir(os.path.dirname(values_path) or "."):
            vals.tofile(values_path)
        return vals, avg


def BFS32(file_path: str, src_vertex: int = 1, n_runs: int = 1, n_neighbor_gpus: int = 0,
          hbm_budget_bytes: Optional[int] = None, values_path: str = "results/values.bin"):
    return _driver(file_path, "csr", False, "bfs", src_vertex, n_runs, n_neighbor_gpus,
                   hbm_budget_bytes, values_path)


def CC32(file_path: str, n_runs: int = 1, n_neighbor_gpus: int = 0,
         hbm_budget_bytes: Optional[int] = None, values_path: str = "results/values.bin"):
    return _driver(file_path, "csr", False, "cc", 0, n_runs, n_neighbor_gpus,
                   hbm_budget_bytes, values_path)


def SSSP32(file_path: str, src_vertex: int = 1, n_runs: int = 1, n_neighbor_gpus: int = 0,
           hbm_budget_bytes: Optional[int] = None, values_path: str = "results/values.bin"):
    fmt = "wcsr" if file_path.endswith(".wcsr") else "csr"
    return _driver(file_path, fmt, True, "sssp", src_vertex, n_runs, n_neighbor_gpus,
                   hbm_budget_bytes, values_path)


def PR32(file_path: str, n_runs: int = 1, n_neighbor_gpus: int = 0,
         hbm_budget_bytes: Optional[int] = None, values_path: str = "results/values.bin"):
    return _driver(file_path, "csc", False, "pr_pull", 0, n_runs, n_neighbor_gpus,
                   hbm_budget_bytes, values_path)


def PR32_PUSH(file_path: str, n_runs: int = 1, n_neighbor_gpus: int = 0,
              hbm_budget_bytes: Optional[int] = None, values_path: str = "results/values.bin"):
    return _driver(file_path, "csr", False, "pr_push", 0, n_runs, n_neighbor_gpus,
                   hbm_budget_bytes, values_path)


def values_checksum(values: np.ndarray) -> int:
    """Order-independent checksum of a u32 value array, as thv_batch_run
    computes per source: sum over v of splitmix64((v << 32) | value) mod 2^64."""
    v = np.asarray(values, dtype=np.uint64)
    x = (np.arange(len(v), dtype=np.uint64) << np.uint64(32)) | v
    with np.errstate(over="ignore"):
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
        return int(x.sum(dtype=np.uint64))


def link_bandwidth(device: int = 0, nbytes: int = 1 << 30):
    """(pinned memcpy H2D GB/s, zero-copy streaming read GB/s) of the host link."""
    lib = load_library()
    mc, zc = ctypes.c_double(), ctypes.c_double()
    _check(lib.thv_link_bandwidth(device, nbytes, ctypes.byref(mc), ctypes.byref(zc)),
           "thv_link_bandwidth")
    return mc.value, zc.value


def now() -> float:
    return time.perf_counter()
