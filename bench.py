#!/usr/bin/env python
"""Benchmarks of the out-of-HBM frontier engine on one B200, every config.

Headline (the JSON line's value): config 2's SSSP.  Directed RMAT scale 24,
edge factor 16 (a=.57, b=.19, c=.19), self-loops and duplicates removed, ids
permuted, WCSR with weights in [1,64]; the HBM edge budget holds 40% of the
edge bytes and the rest is read zero-copy from pinned host memory.  A step
is one SSSP from source 1, bit-exact against the CPU oracle.

The default N=1 run also measures every other config and reports each under
"extra", each with its own parity check, clocks and (C1-C3) roofline:
  c2_sssp_unpacked  the same SSSP with 8-byte {dst, w} edges (packing off),
                    so 60% of the edges cross the host link as config 2 meant
  c2_cc             CC by min-label propagation on the symmetrised graph,
                    40% budget (the reference's method); c2_cc_union_find is
                    the sampling union-find the engine uses by default on
                    symmetric graphs (same labels)
  c1_bfs            BFS, RMAT scale 20, fully resident, source 1
  c3_pr_pull/push   PageRank on RMAT scale 26 (CSC / CSR), 2 GiB HBM edge
                    budget, 20 iterations, every vertex within 1e-6 relative
                    of the FP64 oracle
  c4_bfs/c4_sssp    1,024 seeded sources on RMAT scale 26 in groups of 64
                    vs single-source runs; the first group's 64 checksums
                    equal those of single runs
  c5                a short serving sweep (3 arrival rates) on RMAT scale 26,
                    edge factor 48, served vs the same stream measured one
                    query at a time; every answer equals its single run

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--workload c2|c1|c2cc|c3|c3push|c4|c5] [--no-extra]

value: whole-job GTEPS = traversed edges (sum of out-degrees of the vertices
the source reaches, each counted once) / device time, summed over ranks
(weak scaling: every rank runs its own replica; the path does not shard).
e2e: the same metric through the C ABI with a host output buffer, host
wall-clock, device->host copy of the values inside the timed region.
--impl reference: the CPU oracle (OpenMP, all host threads) on the same
workload -- the reference has no CPU implementation of this path.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 0x54484592
FALLBACK_HBM_GBS = 6650.0
PCIE_GEN5_X16_GBS = 64.0     # spec figure per direction, for context beside the measured link
PR_RTOL = 1e-6               # PageRank: max per-vertex relative error vs the FP64 oracle
TRAFFIC_TABLE = os.path.join(ROOT, "profiles", "ncu_traffic.json")
L2_NOTE = ("inputs larger than L2 (>= 64 MB of edges); the GPU arm also writes 256 MiB "
           "between timed steps, outside the events")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def measured_traffic(key):
    """DRAM read+write bytes and host-link read bytes per launch of the
    dominant kernel, from an ncu capture of exactly this workload (the
    table in profiles/ncu_traffic.json, each entry with its command);
    (None, None, None) when this workload was not captured."""
    try:
        table = json.load(open(TRAFFIC_TABLE))
    except (OSError, ValueError):
        return None, None, None
    e = table.get(key)
    if not e:
        return None, None, None
    return (int(e["dram_read_bytes"] + e["dram_write_bytes"]),
            int(e["sysmem_read_sectors"] * 32) if e.get("sysmem_read_sectors") is not None else None,
            e)


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2",
                    choices=["c1", "c2", "c2cc", "c3", "c3push", "c4", "c5"])
    ap.add_argument("--edge-factor", type=int, default=0, help="override the edge factor")
    ap.add_argument("--rates", default="", help="c5: comma-separated arrival rates (queries/s)")
    ap.add_argument("--sssp-delta", type=int, default=0, help="c4: batched SSSP window width")
    ap.add_argument("--queries", type=int, default=0,
                    help="c4: batched sources (default 1024); c5: queries per rate (default 96, "
                         "256 at the top rate)")
    ap.add_argument("--group-min", type=int, default=0,
                    help="c5: queue depth from which the server runs batched groups (0 = default)")
    ap.add_argument("--join-window", type=int, default=0,
                    help="c5: iterations a running group admits arrivals (0 = the server's "
                         "default, 0xFFFFFFFF = its whole life)")
    ap.add_argument("--groups-per-algo", type=int, default=0,
                    help="c5: batched groups of one algorithm on the device at once (0 = default)")
    ap.add_argument("--scale", type=int, default=0, help="override the workload's scale")
    ap.add_argument("--source", type=int, default=1, help="BFS/SSSP source vertex")
    ap.add_argument("--budget-frac", type=float, default=-1.0,
                    help="override the HBM edge budget as a fraction of edge bytes")
    ap.add_argument("--no-extra", action="store_true", help="headline workload only")
    ap.add_argument("--edge-packing", type=int, default=1, choices=[0, 1],
                    help="weighted graphs: 4-byte packed edges (1) or 8-byte {dst, w} (0)")
    ap.add_argument("--label-propagation", action="store_true",
                    help="c2cc: min-label propagation instead of union-find")
    ap.add_argument("--only", default="", help="comma-separated extra sections to run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--time-guard-s", type=float, default=600.0,
                    help="skip the remaining extra sections once the run is this old")
    return ap.parse_args(argv)


WORKLOADS = {
    "c1": dict(algo="bfs", scale=20, ef=16, fmt="csr", sym=False, frac=1.0),
    "c2": dict(algo="sssp", scale=24, ef=16, fmt="wcsr", sym=False, frac=0.4),
    "c2cc": dict(algo="cc", scale=24, ef=16, fmt="csr", sym=True, frac=0.4),
    "c3": dict(algo="pr_pull", scale=26, ef=16, fmt="csc", sym=False, budget=2 << 30),
    "c3push": dict(algo="pr_push", scale=26, ef=16, fmt="csr", sym=False, budget=2 << 30),
}


def budget_desc(wl):
    if "budget" in wl:
        return f"{wl['budget']} bytes"
    return f"{int(round(wl['frac'] * 100))}% of the format's edge bytes"


def traffic_key(wl, packed=True, label_propagation=False):
    """Name of a workload in the traffic table: algorithm (CC: method),
    scale, format, budget, edge storage."""
    algo = wl["algo"]
    if algo == "cc":
        algo = "cc_lp" if label_propagation or not wl["sym"] else "cc_uf"
    budget = f"{wl['budget'] >> 20}MiB" if "budget" in wl else f"{int(round(wl['frac'] * 100))}pct"
    return f"{algo}_rmat{wl['scale']}_{wl['fmt']}{'_sym' if wl['sym'] else ''}_{budget}" + \
        ("" if packed or wl["fmt"] != "wcsr" else "_unpacked")


def workload_config(wl, source, gpus):
    """The config dict both arms print (keys that describe the workload only)."""
    return {"workload": f"{wl['algo']} rmat{wl['scale']} ef{wl['ef']} {wl['fmt']} "
                        f"hbm-budget {budget_desc(wl)}",
            "scale": wl["scale"], "edge_factor": wl["ef"], "format": wl["fmt"],
            "symmetric": wl["sym"], "hbm_edge_budget": budget_desc(wl),
            "source": source if wl["algo"] in ("bfs", "sssp") else None,
            "pr_iterations": 20 if wl["algo"].startswith("pr") else None,
            "parallelism": f"replicas x{gpus}", "l2": L2_NOTE}


class Dist:
    def __init__(self, n):
        self.n = n
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist
            import datetime
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8], float(f[3])))
            except ValueError:
                pass
        os.unlink(self.path)
        if not rows:
            return None
        reasons = []
        for i, name in [(2, "hw_slowdown"), (3, "hw_thermal_slowdown"), (4, "sw_thermal_slowdown"),
                        (5, "sw_power_cap")]:
            if any(r[i].lower().startswith("active") for r in rows):
                reasons.append(name)
        busy = [r[0] for r in rows if r[6] > 250] or [r[0] for r in rows]
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(off, vals, nv, vb, res, esz, algo, n_iters=1, list_deg=0):
    """Per-run bytes a work-optimal run must move, split HBM / host link.

    BFS/SSSP: every reached vertex is expanded once: 16 B of offsets and a
    4 B value write, its adjacency (esz per edge as stored: 4 B for packed
    weighted edges; over the host link when its
    block is not resident and the list is not in the small-list cache,
    0 < deg < list_deg) and a 4 B value probe per edge.  CC/PR: every
    vertex once per iteration (CC: the synchronous label-propagation sweep
    count is not fixed, so the bytes of ONE full sweep are used -- a lower
    bound)."""
    deg = np.diff(off.astype(np.int64))
    if algo in ("bfs", "sssp"):
        mask = vals < nv + 1
    else:
        mask = np.ones(nv, bool)
    blk = np.searchsorted(vb.astype(np.int64), np.arange(nv), side="right") - 1
    resident_v = res[blk] | ((deg > 0) & (deg < list_deg))
    d = deg[mask]
    r = resident_v[mask]
    per_edge_probe = 4 if algo != "pr_push" else 8
    link = int((d[~r] * esz).sum())
    hbm = int((d[r] * esz).sum() + d.sum() * per_edge_probe + mask.sum() * (16 + 4))
    return hbm * n_iters, link * n_iters, int(d.sum())


UF_SAMPLE = 2  # neighbours each vertex unions with first (union-find CC)


def algorithmic_bytes_cc_uf(off, labels, nv, vb, res, esz, list_deg):
    """Bytes sampling union-find CC must move on a symmetric graph: offsets
    and label init/flatten per vertex (16 + 12 B), the first UF_SAMPLE
    neighbours of every vertex and the rest of the lists of vertices outside
    the highest-degree vertex's component, each edge with two 4 B label
    probes; adjacency over the link where its block is on the host and the
    list is not in the small-list cache."""
    deg = np.diff(off.astype(np.int64))
    hub = int(np.argmax(deg))
    outside = labels != labels[hub]
    edges_v = np.minimum(deg, UF_SAMPLE) + np.where(outside, np.maximum(deg - UF_SAMPLE, 0), 0)
    blk = np.searchsorted(vb.astype(np.int64), np.arange(nv), side="right") - 1
    resident_v = res[blk] | ((deg > 0) & (deg < list_deg))
    link = int((edges_v[~resident_v] * esz).sum())
    hbm = int((edges_v[resident_v] * esz).sum() + edges_v.sum() * 8 + nv * (16 + 12))
    return hbm, link, int(edges_v.sum())


def roofline(b_hbm, b_link, kern_s, hbm_peak, peak_kind, link_mc, link_zc, traffic_key,
             launches_per_step, extra=None):
    """Mixed HBM + host-link roofline of one step: T_roof = B_hbm/HBM + B_link/link."""
    link_peak = max(link_mc, link_zc)
    t_roof = b_hbm / (hbm_peak * 1e9) + b_link / (link_peak * 1e9)
    t_spec = b_hbm / (hbm_peak * 1e9) + b_link / (PCIE_GEN5_X16_GBS * 1e9)
    dram, link_t, entry = measured_traffic(traffic_key)
    per = max(int(launches_per_step), 1)
    r = {"bound": "hbm", "unit": "GB/s",
         "achieved": (b_hbm + b_link) / kern_s / 1e9,
         "peak": (b_hbm + b_link) / t_roof / 1e9,
         "frac": t_roof / kern_s,
         "frac_vs_pcie_gen5_spec": t_spec / kern_s,
         "traffic": None if dram is None else dram * (entry.get("launches_per_step", 1)),
         "link_traffic": None if link_t is None else link_t * (entry.get("launches_per_step", 1)),
         "traffic_source": (f"ncu capture of this workload: {entry['command']}" if entry else
                            "not captured at this size (null)"),
         "algorithmic_hbm_bytes": b_hbm, "algorithmic_link_bytes": b_link,
         "hbm_peak_gbs": hbm_peak, "hbm_peak_kind": peak_kind,
         "link_peak_gbs": link_peak, "link_memcpy_gbs": link_mc, "link_zerocopy_gbs": link_zc,
         "pcie_gen5_x16_spec_gbs": PCIE_GEN5_X16_GBS,
         "kernel_ms": kern_s * 1e3, "launches_per_step": per,
         "note": ("mixed bound: peak = bytes / (B_hbm/HBM + B_link/link), with HBM of measured "
                  "and the link's measured pinned-memcpy or zero-copy rate; frac = T_roof / T")}
    if extra:
        r.update(extra)
    return r


class Bench:
    """Per-process state shared by the measurements: device, stream, L2
    flush buffer, peaks and the host-link rates."""

    def __init__(self, args, dist):
        import torch
        import thievory_b200 as T

        self.torch, self.T, self.args, self.dist = torch, T, args, dist
        self.dev = dist.local
        torch.cuda.set_device(self.dev)
        T.load_library()
        self.hbm_peak, self.peak_kind = peaks()
        self.link_mc, self.link_zc = T.link_bandwidth(self.dev, 1 << 30)
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{self.dev}")
        self.stream = torch.cuda.Stream(device=self.dev)
        self.sptr = self.stream.cuda_stream
        self.t_start = time.perf_counter()

    def gen(self, wl):
        return self.T.Graph.generate_rmat(wl["scale"], wl["ef"], seed=SEED, symmetric=wl["sym"],
                                          fmt=wl["fmt"], device=self.dev)

    @staticmethod
    def plan(g, wl, algo=None):
        algo = algo or wl["algo"]
        budget = wl["budget"] if "budget" in wl else int(wl["frac"] * g.ne * g.esz)
        # PageRank reads whole blocks: no small-list cache
        return budget, g.plan(budget, small_list_degree=1 if algo.startswith("pr") else 0)

    def timed(self, g, algo, k, w, run_kw):
        """w warm-up runs, then k runs each bracketed by CUDA events on the
        launching stream, a 256 MiB write between them (outside the events),
        clocks sampled throughout, barrier + synchronize on both sides."""
        torch, dist = self.torch, self.dist
        for _ in range(w):
            g.run(algo, source=self.args.source, want_values=False, stream=self.sptr, **run_kw)
        ck = Clocks(self.dev).start()
        dist.barrier()
        torch.cuda.synchronize(self.dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        lib_ms, launches, link_bytes, hbm_bytes = [], 0, 0, 0
        with torch.cuda.stream(self.stream):
            for i in range(k):
                self.flush.zero_()
                ev[i][0].record(self.stream)
                _, st = g.run(algo, source=self.args.source, want_values=False, stream=self.sptr,
                              **run_kw)
                ev[i][1].record(self.stream)
                lib_ms.append(st["device_ms"])
                launches += st["kernel_launches"]
                link_bytes += st["link_edge_bytes"]
                hbm_bytes += st["hbm_edge_bytes"]
        self.stream.synchronize()
        dist.barrier()
        clocks = ck.stop()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        total_s = dist.max(sum(step_ms) / 1e3)
        return {"total_s": total_s, "step_ms": step_ms, "lib_ms": lib_ms, "launches": launches,
                "link_bytes": link_bytes // k, "hbm_bytes": hbm_bytes // k, "clocks": clocks,
                "k": k}

    def measure(self, wl, k, w, want_e2e=False, cpu=True, run_kw=None, traffic_key=None,
                graph=None, keep=False, label=""):
        """One single-source / whole-graph workload: timing, roofline, the
        oracle's answer on the host (checked equal; its time is the CPU
        baseline), optionally e2e through the C ABI."""
        from oracle import oracle as O

        T, dist, args = self.T, self.dist, self.args
        run_kw = dict(run_kw or {})
        g = graph or self.gen(wl)
        algo = wl["algo"]
        budget, plan = self.plan(g, wl)
        src = args.source
        tm = self.timed(g, algo, k, w, run_kw)
        vals = g.values(algo)
        off, edges, outdeg = g.host_arrays()
        vb, res = g.blocks()
        iters = 20 if algo.startswith("pr") else 1
        lcd = 0 if algo.startswith("pr") else plan["small_list_degree"]
        union_find = algo == "cc" and g.symmetric and not run_kw.get("label_propagation")
        if union_find:
            b_hbm, b_link, _ = algorithmic_bytes_cc_uf(off, vals, g.nv, vb, res, g.mem_esz, lcd)
        else:
            b_hbm, b_link, trav = algorithmic_bytes(off, vals if algo in ("bfs", "sssp") else None,
                                                    g.nv, vb, res, g.mem_esz, algo, iters, lcd)
        if algo == "cc" or algo.startswith("pr"):
            trav = g.ne * iters  # edges of the graph, however many were read
        kern_s = statistics.mean(tm["lib_ms"]) / 1e3
        out = {
            "value": dist.n * trav * tm["k"] / tm["total_s"] / 1e9, "unit": "GTEPS",
            "ms_per_step": tm["total_s"] * 1e3 / tm["k"], "steps": tm["k"], "warmup": w,
            "traversed_edges": trav, "clocks": tm["clocks"],
            "gpu_launches": tm["launches"],
            "plan": {k_: plan[k_] for k_ in ("num_blocks", "resident_blocks", "resident_edge_bytes",
                                             "host_edge_bytes", "small_list_degree",
                                             "small_list_bytes", "small_list_vertices")},
            "storage": {"format_edge_bytes": g.esz, "stored_edge_bytes": g.mem_esz,
                        "packed_weight_bits": g.weight_bits, "budget_bytes": budget},
            "roofline": roofline(b_hbm, b_link, kern_s, self.hbm_peak, self.peak_kind, self.link_mc,
                                 self.link_zc, traffic_key, tm["launches"] / tm["k"],
                                 {"actual_link_bytes_per_step": tm["link_bytes"],
                                  "actual_hbm_edge_bytes_per_step": tm["hbm_bytes"]}),
        }
        if want_e2e:
            host = self.torch.empty(g.nv * (2 if algo.startswith("pr") else 1),
                                    dtype=self.torch.int32).pin_memory()
            hv = host.numpy().view(np.float64 if algo.startswith("pr") else np.uint32)
            wall = []
            for _ in range(k):
                t0 = time.perf_counter()
                _, st = g.run(algo, source=src, out=hv, stream=self.sptr, **run_kw)
                wall.append(time.perf_counter() - t0)
            tw = dist.max(sum(wall))
            out["e2e"] = {"value": dist.n * trav * k / tw / 1e9, "unit": "GTEPS",
                          "h2d_bytes_per_step": int(st["link_edge_bytes"] + st["h2d_bytes"]),
                          "d2h_bytes_per_step": int(st["d2h_bytes"]),
                          "note": "h2d = zero-copy edge bytes read over the host link"}
            if algo in ("bfs", "sssp", "cc"):
                assert np.array_equal(hv, vals), "e2e values differ from device run"
        if cpu and dist.rank == 0 and dist.n == 1:
            L = O.lib()
            P = lambda a: None if a is None else a.ctypes.data  # noqa: E731
            t0 = time.perf_counter()
            if algo in ("bfs", "sssp", "cc"):
                cv = np.empty(g.nv, np.uint32)
                if algo == "sssp":
                    L.thvo_sssp_par(g.nv, P(off), P(edges), None, 2, src, P(cv))
                elif algo == "bfs":
                    L.thvo_bfs_par(g.nv, P(off), P(edges), 1, src, P(cv))
                else:
                    L.thvo_cc_par(g.nv, P(off), P(edges), 1, P(cv))
                dt = time.perf_counter() - t0
                assert np.array_equal(cv, vals), f"{label or algo}: GPU result differs from the CPU oracle"
                out["check"] = (f"all {g.nv} values bit-exact vs the CPU oracle "
                                f"({'Dijkstra-equivalent label-correcting' if algo == 'sssp' else algo})")
                out["oracle_values"] = cv
            else:
                # the FP64 oracle over the in-edges (CSC); a CSR graph's is
                # supplied by the caller (the transpose of the same graph)
                cv = np.empty(g.nv, np.float64)
                L.thvo_pagerank_csc(g.nv, P(off), P(edges), P(outdeg), 20, 0.85, P(cv))
                dt = time.perf_counter() - t0
                out["oracle_values"] = cv
            out["cpu_baseline"] = {"value": trav / dt / 1e9, "unit": "GTEPS", "cores": O.threads(),
                                   "kind": "port",
                                   "sample": f"one full run of this workload on the host "
                                             f"(OpenMP oracle, {dt:.2f} s)"}
        out["values"] = vals
        if keep:
            out["graph"] = g
        elif graph is None:
            g.close()
        return out

    def elapsed(self):
        return time.perf_counter() - self.t_start


def public(d, drop=("values", "oracle_values", "graph")):
    return {k: v for k, v in d.items() if k not in drop}


def pr_check(gpu, ref, label):
    rel = float(np.max(np.abs(gpu - ref) / np.abs(ref)))
    assert rel <= PR_RTOL, f"{label}: PageRank max relative error {rel:.3e} > {PR_RTOL}"
    return rel


def run_headline(b, args):
    """Config 2 SSSP (the line's value) and, with extras, the rest of config 2."""
    wl = dict(WORKLOADS[args.workload])
    if args.scale:
        wl["scale"] = args.scale
    if args.budget_frac >= 0:
        wl.pop("budget", None)
        wl["frac"] = args.budget_frac
    key = traffic_key(wl, packed=bool(args.edge_packing), label_propagation=args.label_propagation)
    keep = args.workload == "c2" and not args.no_extra and b.dist.world == 1
    graph = None
    if not args.edge_packing:
        graph = b.gen(wl)
        graph.set_edge_packing(False)
    run_kw = {"label_propagation": True} if args.label_propagation else None
    main = b.measure(wl, args.steps, args.warmup, want_e2e=True, cpu=not args.no_cpu,
                     traffic_key=key, keep=keep, graph=graph, run_kw=run_kw)
    if graph is not None and not keep:
        graph.close()
    if wl["algo"] in ("pr_pull",) and "oracle_values" in main:
        main["check"] = (f"all {len(main['values'])} ranks within "
                         f"{pr_check(main['values'], main['oracle_values'], 'pagerank'):.2e} "
                         f"relative of the FP64 oracle (tolerance {PR_RTOL})")
    extra = {}
    if keep:
        g = main.pop("graph")
        ref_vals = main.get("oracle_values", main["values"])
        # config 2 as it was meant: 8-byte {dst, w} edges, 40% of them resident
        g.set_edge_packing(False)
        up = b.measure(wl, max(3, args.steps // 2), 3, cpu=False, graph=g,
                       traffic_key=traffic_key(wl, packed=False))
        assert np.array_equal(up["values"], ref_vals), "unpacked SSSP differs"
        up["check"] = "all values bit-exact vs the packed run (itself checked vs the CPU oracle)"
        extra["c2_sssp_unpacked"] = public(up)
        g.close()
        # CC: min-label propagation is the reference's method (the CC figure);
        # union-find is the engine's default on symmetric graphs
        wcc = dict(WORKLOADS["c2cc"], scale=wl["scale"])
        gcc = b.gen(wcc)
        lp = b.measure(wcc, args.steps, args.warmup, cpu=not args.no_cpu,
                       run_kw={"label_propagation": True}, graph=gcc,
                       traffic_key=traffic_key(wcc, label_propagation=True), label="cc label propagation")
        lp["algorithm"] = "min-label propagation (the reference's CC method)"
        extra["c2_cc"] = public(lp)
        uf = b.measure(wcc, args.steps, args.warmup, cpu=False, graph=gcc,
                       traffic_key=traffic_key(wcc))
        if "oracle_values" in lp:
            assert np.array_equal(uf["values"], lp["oracle_values"]), "union-find CC differs"
            uf["check"] = "all labels bit-exact vs the CPU oracle (min-label fixed point)"
        uf["algorithm"] = ("sampling union-find (the graph is symmetric): same labels as min-label "
                           "propagation, reads 3% of the edges; GTEPS counts every edge")
        extra["c2_cc_union_find"] = public(uf)
        gcc.close()
    return wl, main, extra


def run_c1(b, args):
    wl = dict(WORKLOADS["c1"])
    m = b.measure(wl, args.steps, args.warmup, want_e2e=True, cpu=not args.no_cpu,
                  traffic_key=traffic_key(wl))
    m["config"] = workload_config(wl, args.source, args.gpus)
    return public(m)


def run_c3(b, args):
    """PageRank pull (CSC) and push (CSR), 20 iterations, both checked at
    every vertex against one FP64 oracle run over the CSC (the CSR is the
    same graph: the generator builds the CSC as its transpose)."""
    k, w = min(args.steps, 3), 3
    out = {}
    wl = dict(WORKLOADS["c3"])
    pull = b.measure(wl, k, w, cpu=not args.no_cpu, traffic_key=traffic_key(wl))
    ref = pull.pop("oracle_values", None)
    if ref is not None:
        pull["check"] = (f"all {len(ref)} ranks after 20 iterations within "
                         f"{pr_check(pull['values'], ref, 'pr_pull'):.2e} relative of the FP64 "
                         f"oracle (tolerance {PR_RTOL})")
    pull["config"] = workload_config(wl, None, args.gpus)
    out["c3_pr_pull"] = public(pull)
    wl = dict(WORKLOADS["c3push"])
    push = b.measure(wl, k, w, cpu=False, traffic_key=traffic_key(wl), keep=True)
    if ref is not None:
        push["check"] = (f"all {len(ref)} ranks after 20 iterations within "
                         f"{pr_check(push['values'], ref, 'pr_push'):.2e} relative of the FP64 "
                         f"oracle (tolerance {PR_RTOL})")
        push["cpu_baseline"] = dict(pull["cpu_baseline"],
                                    sample=pull["cpu_baseline"]["sample"] + "; the same oracle run "
                                    "(pull over the CSC) gives the push ranks")
    push["config"] = workload_config(wl, None, args.gpus)
    g = push.pop("graph")
    out["c3_pr_push"] = public(push)
    return out, g


def run_c4(b, args, g_csr=None):
    """Config 4: 1,024 seeded sources over the non-isolated vertices of
    RMAT scale 26, batched in groups of 64 (one persistent, graph-captured
    launch per group) vs single-source runs of the first group's 64 sources,
    whose checksums must equal the batched ones bit for bit."""
    T = b.T
    scale = args.scale if args.workload == "c4" and args.scale else 26
    n = args.queries or 1024
    out = {}
    for algo, fmt in (("bfs", "csr"), ("sssp", "wcsr")):
        g = g_csr if (algo == "bfs" and g_csr is not None and scale == 26) else \
            T.Graph.generate_rmat(scale, 16, seed=SEED, fmt=fmt, device=b.dev)
        budget = 2 << 30 if args.budget_frac < 0 else int(args.budget_frac * g.ne * g.esz)
        plan = g.plan(budget)
        src = g.pick_sources(n, SEED)
        dl = args.sssp_delta if algo == "sssp" else 0
        g.batch_run(algo, src[:64], want_values=False, sssp_delta=dl, tune=True)  # tunes, warms up
        ck = Clocks(b.dev).start()
        _, sums, bst = g.batch_run(algo, src, want_values=False, sssp_delta=dl, tune=True)
        clocks = ck.stop()
        tuned = g.batch_tuned(algo)
        nplain = min(64, n)
        plain_ms, plain_bytes = [], []
        for i, s_ in enumerate(src[:nplain]):
            _, st = g.run(algo, source=int(s_), want_values=False, checksum=True)
            plain_ms.append(st["device_ms"])
            plain_bytes.append(st["hbm_edge_bytes"] + st["link_edge_bytes"])
            assert st["checksum"] == int(sums[i]), f"c4 {algo} source {s_} differs"
        qps_b = b.dist.n * len(src) / (b.dist.max(bst["device_ms"]) / 1e3)
        qps_p = b.dist.n * 1e3 / b.dist.max(statistics.mean(plain_ms))
        out[f"c4_{algo}"] = {
            "batched_qps": qps_b, "plain_qps": qps_p, "speedup": qps_b / qps_p,
            "sssp_delta": dl, "batched_ms_total": bst["device_ms"],
            "plain_ms_mean": statistics.mean(plain_ms), "queries": len(src),
            "groups": (len(src) + 63) // 64, "batched_iterations": bst["iterations"],
            "batched_launches": bst["kernel_launches"], "launch_config": tuned,
            "batched_link_bytes": bst["link_edge_bytes"],
            "batched_edge_bytes": bst["hbm_edge_bytes"] + bst["link_edge_bytes"],
            "plain_form_edge_bytes": statistics.mean(plain_bytes) * len(src),
            "clocks": clocks,
            "config": {"workload": f"{algo} rmat{scale} ef16 {fmt}, HBM edge budget {budget} bytes, "
                                   f"{len(src)} seeded sources, groups of 64",
                       "resident_edge_bytes": plan["resident_edge_bytes"],
                       "host_edge_bytes": plan["host_edge_bytes"]},
            "check": (f"the first group's {nplain} sources: single-run checksum == batched checksum "
                      f"(sum over v of splitmix64(v<<32|value))"),
            "timing": "batched: device time of all groups (CUDA events); plain: mean device time "
                      "of the single runs"}
        g.close()
    return out


def stream_plain(g, algos, src, arr):
    """The stream run one query at a time on the plain kernels: each query
    starts at its arrival or when the previous one finishes; host wall
    clock, as the server's latencies."""
    t0 = time.perf_counter()
    lat, sums = [], []
    for i, (a, s_) in enumerate(zip(algos, src)):
        target = t0 + arr[i] - arr[0]
        d = target - time.perf_counter()
        if d > 0:
            time.sleep(d)
        _, st = g.run(a, source=int(s_), want_values=False, checksum=True)
        lat.append(time.perf_counter() - target)
        sums.append(st["checksum"])
    return len(src) / (time.perf_counter() - t0), np.array(lat) * 1e3, sums


def stream_served(T, g, algos, src, arr, group_min, join_window=0, groups_per_algo=0):
    with T.Server(g, max_slots=64, group_min=group_min, join_window=join_window,
                  groups_per_algo=groups_per_algo) as sv:
        t0 = time.perf_counter()
        tickets = []
        for i, (a, s_) in enumerate(zip(algos, src)):
            d = t0 + arr[i] - arr[0] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets.append(sv.submit(a, int(s_), want_values=False))
        stats = [sv.wait(t, timeout_ms=600000)[1] for t in tickets]
        t1 = time.perf_counter()
    return len(src) / (t1 - t0), stats


def run_c5(b, args):
    """Config 5 (scaled to the box; the scale-30 graph needs ~206 GB CSR
    of pinned host memory): a Poisson stream, 80% BFS / 20% SSSP, sources
    uniform over non-isolated vertices, served with continuous batching vs
    the same stream measured one query at a time on the plain kernels.
    Every served answer's checksum equals the plain run's."""
    T = b.T
    scale = args.scale if args.workload == "c5" and args.scale else 26
    ef = args.edge_factor or 48
    frac = args.budget_frac if args.budget_frac >= 0 else 0.58
    n_low = args.queries or 96
    n_top = args.queries or 256  # saturation: enough queries for steady state
    g = T.Graph.generate_rmat(scale, ef, seed=SEED, fmt="wcsr", device=b.dev)
    # HBM budget: frac of the graph's CSR bytes (4 per edge), as ~120 GB of
    # the ~206 GB CSR at scale 30 / edge factor 48
    plan = g.plan(int(frac * g.ne * 4))
    nmax = max(n_low, n_top)
    src_all = g.pick_sources(nmax, SEED)
    algos_all = ["sssp" if i % 5 == 0 else "bfs" for i in range(nmax)]
    # warm-up outside the sweep: tune the batched-group kernels the server
    # uses for deep queues (cached in-process) and allocate their state
    for a in ("bfs", "sssp"):
        g.batch_run(a, src_all[:64], want_values=False, tune=True)
    probe = [g.run(a, source=int(s_), want_values=False)[1]["device_ms"]
             for a, s_ in zip(algos_all[:10], src_all[:10])]
    cap = 1e3 / statistics.mean(probe)  # plain capacity estimate, queries/s
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [cap, 4 * cap, 32 * cap]
    rng = np.random.default_rng(SEED)
    sweep, answers = [], {}
    ck = Clocks(b.dev).start()
    for ri, rate in enumerate(rates):
        n = n_top if ri == len(rates) - 1 else n_low
        src, algos = src_all[:n], algos_all[:n]
        arr = np.cumsum(rng.exponential(1.0 / rate, n))
        pq, plat, psum = stream_plain(g, algos, src, arr)
        for i, x in enumerate(psum):
            assert answers.setdefault(i, x) == x, "plain stream answers differ between rates"
        sq, stats = stream_served(T, g, algos, src, arr, args.group_min, args.join_window,
                                  args.groups_per_algo)
        for i, st in enumerate(stats):
            assert st["checksum"] == answers[i], f"c5 query {i} ({algos[i]} {src[i]}) differs"
        slat = np.array([st["latency_ms"] for st in stats])
        modes = [st["grouped"] for st in stats]
        joined = sum(st["joined"] for st in stats)
        sweep.append({"rate_qps": rate, "queries": n, "served_qps": sq, "plain_qps": pq, "speedup": sq / pq,
                      "served_p50_ms": float(np.percentile(slat, 50)),
                      "served_p99_ms": float(np.percentile(slat, 99)),
                      "plain_p50_ms": float(np.percentile(plat, 50)),
                      "plain_p99_ms": float(np.percentile(plat, 99)),
                      "served_modes": {"slot": modes.count(0), "group": modes.count(1),
                                       "alone": modes.count(2), "joined_while_running": joined}})
    clocks = ck.stop()
    g.close()
    return {"sweep": sweep, "clocks": clocks,
            "plain_single_ms_probe": statistics.mean(probe),
            "check": "every served answer's checksum == the plain run's (both streams, every rate)",
            "timing": "host wall clock from the first arrival to the last answer; latency = answer - "
                      "arrival; the plain stream is measured, one query at a time",
            "config": {"workload": f"c5 serving rmat{scale} ef{ef} wcsr, HBM edge budget "
                                   f"{int(round(frac * 100))}% of the CSR bytes, 80% BFS / 20% SSSP, "
                                   f"Poisson arrivals: {n_low} per rate, {n_top} at the top rate",
                       "resident_edge_bytes": plan["resident_edge_bytes"],
                       "host_edge_bytes": plan["host_edge_bytes"]}}


def run_reference(args, dist):
    """CPU oracle (the reference has no CPU path) on the same workload."""
    from oracle import oracle as O

    wl = dict(WORKLOADS[args.workload if args.workload in WORKLOADS else "c2"])
    if args.scale:
        wl["scale"] = args.scale
    if args.budget_frac >= 0:
        wl.pop("budget", None)
        wl["frac"] = args.budget_frac
    # all host cores: torchrun sets OMP_NUM_THREADS=1 for every rank, and
    # here rank 0 alone does the work
    O.set_threads(len(os.sched_getaffinity(0)))
    g = O.rmat(wl["scale"], wl["ef"], seed=SEED, symmetric=wl["sym"], weighted=wl["algo"] == "sssp")
    algo = wl["algo"]
    if algo.startswith("pr"):
        csc = O.transpose(g)
    fn = {"sssp": lambda: O.sssp(g, args.source, parallel=True),
          "bfs": lambda: O.bfs(g, args.source, parallel=True),
          "cc": lambda: O.cc(g, parallel=True),
          "pr_pull": lambda: O.pagerank_csc(*csc, 20),
          "pr_push": lambda: O.pagerank_csc(*csc, 20)}[algo]
    for _ in range(args.warmup):
        vals = fn()
    t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        vals = fn()
        t.append(time.perf_counter() - t0)
    trav = O.reached_edges(g, vals) if algo in ("bfs", "sssp") else g.ne * (20 if algo.startswith("pr") else 1)
    value = trav / statistics.mean(t) / 1e9
    return wl, value, statistics.mean(t) * 1e3, O.threads()


def main():
    args = parse()
    dist = Dist(args.gpus)
    if args.impl == "reference":
        if dist.rank != 0:
            dist.close()
            return
        wl, value, ms, cores = run_reference(args, dist)
        line = {"metric": f"GTEPS ({wl['algo']})", "value": value, "unit": "GTEPS", "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32"
                if not wl["algo"].startswith("pr") else "f64",
                "data": "synthetic (seeded RMAT a=.57 b=.19 c=.19, dedup, no self-loops, permuted ids)",
                "config": workload_config(wl, args.source, args.gpus),
                "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": cores, "kind": "port",
                                 "sample": f"one full {wl['algo']} run per step on the host (OpenMP "
                                           f"oracle; the reference has no CPU implementation)"},
                "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        dist.close()
        return
    b = Bench(args, dist)
    if args.workload in ("c4", "c5"):
        out = run_c4(b, args) if args.workload == "c4" else run_c5(b, args)
        if dist.rank == 0:
            print(json.dumps({"workload": args.workload, "n_gpus": args.gpus, **out},
                             default=float))
        dist.close()
        return
    wl, m, extra = run_headline(b, args)
    sections = ["c1", "c3", "c4", "c5"] if args.workload == "c2" and not args.no_extra else []
    if args.only:
        sections = [s for s in sections if s in args.only.split(",")]
    if dist.world > 1:
        sections = []  # replicas: the extra configs are measured at N=1
    g_csr = None
    for s in sections:
        if b.elapsed() > args.time_guard_s:
            extra[s] = {"skipped": f"time guard: the run was {b.elapsed():.0f} s old"}
            continue
        t0 = time.perf_counter()
        if s == "c1":
            extra["c1_bfs"] = run_c1(b, args)
        elif s == "c3":
            r, g_csr = run_c3(b, args)
            extra.update(r)
        elif s == "c4":
            extra.update(run_c4(b, args, g_csr))
            g_csr = None
        elif s == "c5":
            extra["c5"] = run_c5(b, args)
        extra.setdefault("section_seconds", {})[s] = round(time.perf_counter() - t0, 1)
    if g_csr is not None:
        g_csr.close()
    if dist.rank == 0:
        line = {
            "metric": f"GTEPS ({wl['algo']})", "value": m["value"], "unit": "GTEPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32" if not wl["algo"].startswith("pr") else "f32",
            "data": "synthetic (seeded RMAT a=.57 b=.19 c=.19, dedup, no self-loops, permuted ids)",
            "config": workload_config(wl, args.source, args.gpus),
            "plan": m["plan"], "edge_storage": m["storage"],
            "traversed_edges_per_step": m["traversed_edges"],
            "roofline": m["roofline"], "gpu_launches": m["gpu_launches"],
            "clocks": m["clocks"], "e2e": m.get("e2e"), "check": m.get("check"),
        }
        if "cpu_baseline" in m:
            line["cpu_baseline"] = m["cpu_baseline"]
        if extra:
            line["extra"] = extra
        line["run_seconds"] = round(b.elapsed(), 1)
        print(json.dumps(line, default=float))
    dist.close()


if __name__ == "__main__":
    main()
