#!/usr/bin/env python
"""Headline benchmark: GTEPS of the out-of-HBM frontier engine on one B200.

Default workload (N=1): directed RMAT scale 24, edge factor 16 (a=.57,
b=.19, c=.19), self-loops/duplicates removed, ids permuted, WCSR with
weights in [1,64]; the HBM edge budget holds 40% of the edge bytes, the rest
is read zero-copy from pinned host memory.  A step is one SSSP from source 1
(bit-exact distances).  The second algorithm of the same configuration, CC
(min-label propagation) on the symmetrised graph with the same 40% budget,
is reported under "extra".

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
                  [--workload c2|c1|c3]

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


# DRAM and host-link (sysmem) bytes per launch of the dominant kernel, from the
# ncu captures summarised in profiles/ (minq_sssp_rmat22_wcsr_packed_hbm40.md,
# minprop_cc_rmat22_sym_hbm40.md, minprop_bfs_rmat20_resident.md,
# pr_pull_rmat22_csc_hbm47.md).  Captures
# made on a smaller graph are scaled to the bench size by edge count (the
# traffic of these kernels grows with the edges traversed).
NCU_TRAFFIC = {
    "sssp": dict(scale=22, ne=65241959, dram=597834496 + 83409920, sysmem=3283365 * 32),
    "cc": dict(scale=22, ne=128306542, dram=392704512 + 69563648, sysmem=11788847 * 32),
    "bfs": dict(scale=20, ne=16084564, dram=41359616 + 613888, sysmem=0),
    "pr_pull": dict(scale=22, ne=65241959, dram=135399168 + 20317184, sysmem=6104134 * 32, per="iteration"),
}


def traffic_for(algo, scale, ne, iters=1):
    t = NCU_TRAFFIC.get(algo)
    if not t:
        return None, None
    f = ne / t["ne"]
    return int(t["dram"] * f * iters), int(t["sysmem"] * f * iters)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c2cc", "c3", "c4", "c5"])
    ap.add_argument("--edge-factor", type=int, default=0, help="override the edge factor")
    ap.add_argument("--rates", default="", help="c5: comma-separated arrival rates (queries/s)")
    ap.add_argument("--sssp-delta", type=int, default=0, help="c4: batched SSSP window width")
    ap.add_argument("--queries", type=int, default=1024, help="c4: batched sources")
    ap.add_argument("--plain-sample", type=int, default=16, help="c4: single-source runs timed")
    ap.add_argument("--group-min", type=int, default=0,
                    help="c5: queue depth from which the server runs batched groups (0 = default)")
    ap.add_argument("--scale", type=int, default=0, help="override the workload's scale")
    ap.add_argument("--source", type=int, default=1, help="BFS/SSSP source vertex")
    ap.add_argument("--budget-frac", type=float, default=-1.0,
                    help="override the HBM edge budget as a fraction of edge bytes")
    ap.add_argument("--no-extra", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


WORKLOADS = {
    # name: (algo, scale, edge_factor, fmt, symmetric, budget_frac, budget_bytes)
    "c1": dict(algo="bfs", scale=20, ef=16, fmt="csr", sym=False, frac=1.0),
    "c2": dict(algo="sssp", scale=24, ef=16, fmt="wcsr", sym=False, frac=0.4),
    "c2cc": dict(algo="cc", scale=24, ef=16, fmt="csr", sym=True, frac=0.4),
    "c3": dict(algo="pr_pull", scale=26, ef=16, fmt="csc", sym=False, budget=2 << 30),
}


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


def run_ours(args, dist):
    import torch
    import thievory_b200 as T
    from oracle import oracle as O

    dev = dist.local
    torch.cuda.set_device(dev)
    T.load_library()
    hbm_peak, peak_kind = peaks()
    wl = dict(WORKLOADS[args.workload])
    if args.scale:
        wl["scale"] = args.scale
    if args.budget_frac >= 0:
        wl.pop("budget", None)
        wl["frac"] = args.budget_frac

    link_mc, link_zc = T.link_bandwidth(dev, 1 << 30)
    link_peak = max(link_mc, link_zc)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)

    def measure(wl, k, w, want_e2e, want_cpu, run_kw=None):
        run_kw = dict(run_kw or {})
        g = T.Graph.generate_rmat(wl["scale"], wl["ef"], seed=SEED, symmetric=wl["sym"],
                                  fmt=wl["fmt"], device=dev)
        budget = wl.get("budget", int(wl.get("frac", 1.0) * g.ne * g.esz))
        algo = wl["algo"]
        # PageRank reads whole blocks: no small-list cache
        plan = g.plan(budget, small_list_degree=1 if algo.startswith("pr") else 0)
        src = args.source
        sptr = stream.cuda_stream
        for _ in range(w):
            g.run(algo, source=src, want_values=False, stream=sptr, **run_kw)
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
        clocks = Clocks(dev)
        clocks.start()
        dist.barrier()
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        lib_ms, launches, link_bytes, hbm_bytes = [], 0, 0, 0
        with torch.cuda.stream(stream):
            for i in range(k):
                flush.zero_()  # > L2 write between steps (outside the events)
                ev[i][0].record(stream)
                _, st = g.run(algo, source=src, want_values=False, stream=sptr, **run_kw)
                ev[i][1].record(stream)
                lib_ms.append(st["device_ms"])
                launches += st["kernel_launches"]
                link_bytes += st["link_edge_bytes"]
                hbm_bytes += st["hbm_edge_bytes"]
        stream.synchronize()
        dist.barrier()
        ck = clocks.stop()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        total_s = dist.max(sum(step_ms) / 1e3)
        value = dist.n * trav * k / total_s / 1e9
        t_roof = b_hbm / (hbm_peak * 1e9) + b_link / (link_peak * 1e9)
        kern_s = statistics.mean(lib_ms) / 1e3
        # the captured CC kernel is label propagation's; union-find has its own
        dram_t, link_t = traffic_for("cc_uf" if union_find else algo, wl["scale"], g.ne, iters)
        out = {
            "value": value, "ms_per_step": total_s * 1e3 / k, "traversed_edges": trav,
            "plan": plan, "clocks": ck, "gpu_launches": launches,
            "storage": {"format_edge_bytes": g.esz, "stored_edge_bytes": g.mem_esz,
                        "packed_weight_bits": g.weight_bits, "budget_bytes": budget},
            "roofline": {
                "bound": "hbm", "unit": "GB/s",
                "achieved": (b_hbm + b_link) / kern_s / 1e9,
                "peak": (b_hbm + b_link) / t_roof / 1e9,
                "frac": t_roof / kern_s,
                "traffic": dram_t, "link_traffic": link_t,
                "traffic_note": "dram read+write (and host-link sysmem sectors) per launch from an "
                                "ncu capture, scaled by edge count when captured on a smaller graph",
                "algorithmic_hbm_bytes": b_hbm, "algorithmic_link_bytes": b_link,
                "hbm_peak_gbs": hbm_peak, "hbm_peak_kind": peak_kind,
                "link_peak_gbs": link_peak, "link_memcpy_gbs": link_mc, "link_zerocopy_gbs": link_zc,
                "kernel_ms": kern_s * 1e3,
                "actual_link_bytes_per_step": link_bytes // k,
                "actual_hbm_edge_bytes_per_step": hbm_bytes // k,
                "note": "mixed bound: peak = bytes / (B_hbm/HBM + B_link/link); frac = T_roof / T",
            },
        }
        if want_e2e:
            host = torch.empty(g.nv * (2 if algo.startswith("pr") else 1), dtype=torch.int32).pin_memory()
            hv = host.numpy().view(np.float64 if algo.startswith("pr") else np.uint32)
            wall = []
            for _ in range(k):
                t0 = time.perf_counter()
                _, st = g.run(algo, source=src, out=hv, stream=sptr, **run_kw)
                wall.append(time.perf_counter() - t0)
            tw = dist.max(sum(wall))
            out["e2e"] = {"value": dist.n * trav * k / tw / 1e9, "unit": "GTEPS",
                          "h2d_bytes_per_step": int(st["link_edge_bytes"] + st["h2d_bytes"]),
                          "d2h_bytes_per_step": int(st["d2h_bytes"]),
                          "note": "h2d = zero-copy edge bytes read over the host link"}
            if algo in ("bfs", "sssp", "cc"):
                assert np.array_equal(hv, vals), "e2e values differ from device run"
        if want_cpu and dist.rank == 0 and dist.n == 1:
            L = O.lib()
            cv = np.empty(g.nv, np.uint32)
            P = lambda a: None if a is None else a.ctypes.data
            t0 = time.perf_counter()
            if algo == "sssp":
                L.thvo_sssp_par(g.nv, P(off), P(edges), None, 2, src, P(cv))
            elif algo == "bfs":
                L.thvo_bfs_par(g.nv, P(off), P(edges), 1, src, P(cv))
            elif algo == "cc":
                L.thvo_cc_par(g.nv, P(off), P(edges), 1, P(cv))
            elif algo == "pr_pull":
                # bounded sample: 2 of the 20 iterations, checked against the
                # GPU run of the same 2 iterations
                pr_cpu = np.empty(g.nv, np.float64)
                L.thvo_pagerank_csc(g.nv, P(off), P(edges), P(outdeg), 2, 0.85, P(pr_cpu))
            dt = time.perf_counter() - t0
            sample = f"one full {algo} run of this workload on the host"
            work = trav
            if algo in ("bfs", "sssp", "cc"):
                assert np.array_equal(cv, vals), "GPU result differs from the CPU oracle"
            elif algo == "pr_pull":
                gpu2, _ = g.run(algo, pr_iters=2, stream=sptr)
                assert np.max(np.abs(gpu2 - pr_cpu) / np.abs(pr_cpu)) <= 1e-6, "PageRank differs"
                work = 2 * g.ne
                sample = "2 PageRank iterations of this workload on the host"
            out["cpu_baseline"] = {"value": work / dt / 1e9, "unit": "GTEPS", "cores": O.threads(),
                                   "kind": "port",
                                   "sample": f"{sample} (OpenMP oracle, {dt:.2f} s); "
                                             "result checked equal"}
        g.close()
        return out

    main = measure(wl, args.steps, args.warmup, True, not args.no_cpu)
    extra = {}
    if args.workload == "c2" and not args.no_extra:
        cc = measure(dict(WORKLOADS["c2cc"], scale=wl["scale"]), args.steps, args.warmup, False,
                     not args.no_cpu)
        extra["cc_rmat_sym_40pct"] = {k: cc[k] for k in ("value", "ms_per_step", "traversed_edges",
                                                          "roofline", "gpu_launches")}
        extra["cc_rmat_sym_40pct"]["algorithm"] = ("sampling union-find (the graph is symmetric): "
                                                   "same labels as min-label propagation")
        if "cpu_baseline" in cc:
            extra["cc_rmat_sym_40pct"]["cpu_baseline"] = cc["cpu_baseline"]
        lp = measure(dict(WORKLOADS["c2cc"], scale=wl["scale"]), args.steps, args.warmup, False,
                     False, {"label_propagation": True})
        extra["cc_rmat_sym_40pct_label_propagation"] = {
            k: lp[k] for k in ("value", "ms_per_step", "traversed_edges", "roofline", "gpu_launches")}
    return wl, main, extra


def run_batched(args, dist):
    """Config 4: 1,024 seeded sources over the non-isolated vertices, batched
    in groups of 64 (one persistent launch per group) vs single-source runs
    of a sample of the same sources; per-source checksums of the sample must
    match the batched ones bit for bit."""
    import torch
    import thievory_b200 as T

    dev = dist.local
    torch.cuda.set_device(dev)
    T.load_library()
    scale = args.scale or 26
    budget = 2 << 30 if args.budget_frac < 0 else None
    out = {}
    for algo, fmt in (("bfs", "csr"), ("sssp", "wcsr")):
        g = T.Graph.generate_rmat(scale, 16, seed=SEED, fmt=fmt, device=dev)
        g.plan(budget if budget is not None else int(args.budget_frac * g.ne * g.esz))
        src = g.pick_sources(args.queries, SEED)
        dl = args.sssp_delta if algo == "sssp" else 0
        g.batch_run(algo, src[:64], want_values=False, sssp_delta=dl, tune=True)  # tunes, warms up
        _, sums, bst = g.batch_run(algo, src, want_values=False, sssp_delta=dl, tune=True)
        plain_ms, plain_bytes = [], []
        for s_ in src[: args.plain_sample]:
            vals, st = g.run(algo, source=int(s_))
            plain_ms.append(st["device_ms"])
            plain_bytes.append(st["hbm_edge_bytes"] + st["link_edge_bytes"])
            i = int(np.nonzero(src == s_)[0][0])
            assert T.values_checksum(vals) == int(sums[i]), f"{algo} source {s_} differs"
        qps_b = dist.n * len(src) / (dist.max(bst["device_ms"]) / 1e3)
        qps_p = dist.n * 1e3 / dist.max(statistics.mean(plain_ms))
        out[algo] = {"batched_qps": qps_b, "plain_qps": qps_p, "speedup": qps_b / qps_p,
                     "sssp_delta": dl,
                     "batched_ms_total": bst["device_ms"], "plain_ms_mean": statistics.mean(plain_ms),
                     "queries": len(src), "plain_sample": args.plain_sample,
                     "batched_link_bytes": bst["link_edge_bytes"], "batched_iterations": bst["iterations"],
                     # edge bytes read: all groups together vs the plain form
                     # (sampled mean per query x queries)
                     "batched_edge_bytes": bst["hbm_edge_bytes"] + bst["link_edge_bytes"],
                     "plain_form_edge_bytes": statistics.mean(plain_bytes) * len(src),
                     "checked": f"{args.plain_sample} sources: single-run checksum == batched checksum"}
        g.close()
    return scale, out


def run_serving(args, dist):
    """Config 5 (scaled to the box): a Poisson stream, 80% BFS / 20% SSSP,
    sources uniform over non-isolated vertices, served by continuous batching
    vs the same stream run one query at a time with the plain kernels (FIFO
    replay of measured single-query device times on the same arrivals).
    Every served query's checksum must equal its plain run's."""
    import torch
    import thievory_b200 as T

    dev = dist.local
    torch.cuda.set_device(dev)
    T.load_library()
    scale = args.scale or 26
    ef = args.edge_factor or 48
    frac = args.budget_frac if args.budget_frac >= 0 else 0.58
    g = T.Graph.generate_rmat(scale, ef, seed=SEED, fmt="wcsr", device=dev)
    # HBM budget: frac of the graph's CSR bytes (4 per edge), as ~120 GB of
    # the ~206 GB CSR at scale 30 / edge factor 48
    plan = g.plan(int(frac * g.ne * 4))
    n = args.queries
    src = g.pick_sources(n, SEED)
    algos = ["sssp" if i % 5 == 0 else "bfs" for i in range(n)]
    plain_ms, plain_sum = [], []
    for a, s_ in zip(algos, src):
        _, st = g.run(a, source=int(s_), want_values=False, checksum=True)
        plain_ms.append(st["device_ms"])
        plain_sum.append(st["checksum"])
    # warm-up outside the timed sweep: tune the batched-group kernels the
    # server uses for deep queues (cached in-process) and allocate their state
    for a in ("bfs", "sssp"):
        g.batch_run(a, src[:64], want_values=False, tune=True)
    rng = np.random.default_rng(SEED)
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [
        0.5 * 1e3 / statistics.mean(plain_ms), 4e3 / statistics.mean(plain_ms),
        32e3 / statistics.mean(plain_ms)]
    sweep = []
    for rate in rates:
        arr = np.cumsum(rng.exponential(1.0 / rate, n))
        # plain: FIFO replay of the measured service times on these arrivals
        fin, lat = 0.0, []
        for t_a, ms in zip(arr, plain_ms):
            fin = max(fin, t_a) + ms / 1e3
            lat.append(fin - t_a)
        plain_qps = n / (fin - arr[0])
        with T.Server(g, max_slots=64, group_min=args.group_min) as sv:
            t0 = time.perf_counter()
            tickets = []
            for i, (a, s_) in enumerate(zip(algos, src)):
                d = t0 + arr[i] - arr[0] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets.append(sv.submit(a, int(s_), want_values=False))
            stats = [sv.wait(t, timeout_ms=600000)[1] for t in tickets]
            t1 = time.perf_counter()
        for i, st in enumerate(stats):
            assert st["checksum"] == plain_sum[i], f"query {i} ({algos[i]} {src[i]}) differs"
        slat = np.array([st["latency_ms"] for st in stats])
        sweep.append({"rate_qps": rate, "served_qps": n / (t1 - t0),
                      "served_p50_ms": float(np.percentile(slat, 50)),
                      "served_p99_ms": float(np.percentile(slat, 99)),
                      "plain_qps": plain_qps,
                      "plain_p50_ms": float(np.percentile(np.array(lat) * 1e3, 50)),
                      "plain_p99_ms": float(np.percentile(np.array(lat) * 1e3, 99))})
    g.close()
    return scale, ef, frac, plan, sweep, statistics.mean(plain_ms)


def run_reference(args, dist):
    """CPU oracle (the reference has no CPU path) on the same workload."""
    from oracle import oracle as O

    wl = dict(WORKLOADS[args.workload])
    if args.scale:
        wl["scale"] = args.scale
    # all host cores: torchrun sets OMP_NUM_THREADS=1 for every rank, and
    # here rank 0 alone does the work
    O.set_threads(len(os.sched_getaffinity(0)))
    g = O.rmat(wl["scale"], wl["ef"], seed=SEED, symmetric=wl["sym"], weighted=wl["algo"] == "sssp")
    algo = wl["algo"]
    fn = {"sssp": lambda: O.sssp(g, args.source, parallel=True),
          "bfs": lambda: O.bfs(g, args.source, parallel=True),
          "cc": lambda: O.cc(g, parallel=True),
          "pr_pull": lambda: O.pagerank(g, 20)}[algo]
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
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic (seeded RMAT, CPU generator)",
                "config": {"workload": f"{wl['algo']} rmat{wl['scale']} ef{wl['ef']}"},
                "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": cores, "kind": "port",
                                 "sample": f"full {wl['algo']} run per step on the host (OpenMP oracle)"},
                "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        dist.close()
        return
    if args.workload == "c5":
        scale, ef, frac, plan, sweep, plain_mean = run_serving(args, dist)
        if dist.rank == 0:
            top = max(sweep, key=lambda r: r["served_qps"])
            line = {"metric": "queries/s served (continuous batching, 80% BFS / 20% SSSP)",
                    "value": top["served_qps"], "unit": "queries/s", "n_gpus": args.gpus,
                    "steps": args.queries, "warmup": 0, "ms_per_step": 1e3 / top["served_qps"],
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                    "data": "synthetic (seeded RMAT, Poisson arrivals)",
                    "config": {"workload": f"c5 serving rmat{scale} ef{ef} wcsr, HBM edge budget "
                                           f"{int(frac * 100)}% of the CSR bytes, {args.queries} queries per rate",
                               "resident_edge_bytes": plan["resident_edge_bytes"],
                               "host_edge_bytes": plan["host_edge_bytes"],
                               "small_list_cache": {k: plan[k] for k in (
                                   "small_list_degree", "small_list_bytes", "small_list_vertices")}},
                    "plain_mean_ms": plain_mean, "sweep": sweep}
            print(json.dumps(line))
        dist.close()
        return
    if args.workload == "c4":
        scale, out = run_batched(args, dist)
        if dist.rank == 0:
            b = out["bfs"]
            line = {"metric": "queries/s (batched 64-source BFS)", "value": b["batched_qps"],
                    "unit": "queries/s", "n_gpus": args.gpus, "steps": 1, "warmup": 1,
                    "ms_per_step": b["batched_ms_total"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                    "data": "synthetic (seeded RMAT)",
                    "config": {"workload": f"c4 batched BFS/SSSP rmat{scale} ef16, 2 GiB HBM edge budget, "
                                           f"{args.queries} seeded sources, groups of 64"},
                    "extra": out}
            print(json.dumps(line))
        dist.close()
        return
    wl, m, extra = run_ours(args, dist)
    if dist.rank == 0:
        budget_desc = (f"{int(wl['frac'] * 100)}% of the format's edge bytes" if "frac" in wl
                       else f"{wl['budget']} bytes")
        line = {
            "metric": f"GTEPS ({wl['algo']})", "value": m["value"], "unit": "GTEPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded RMAT a=.57 b=.19 c=.19, dedup, no self-loops, permuted ids)",
            "config": {"workload": f"{wl['algo']} rmat{wl['scale']} ef{wl['ef']} {wl['fmt']} "
                                   f"hbm-budget {budget_desc}",
                       "scale": wl["scale"], "edge_factor": wl["ef"], "format": wl["fmt"],
                       "hbm_edge_budget": budget_desc, "source": args.source,
                       "resident_edge_bytes": m["plan"]["resident_edge_bytes"],
                       "host_edge_bytes": m["plan"]["host_edge_bytes"],
                       "small_list_cache": {k: m["plan"][k] for k in (
                           "small_list_degree", "small_list_bytes", "small_list_vertices")},
                       "edge_storage": m["storage"],
                       "traversed_edges_per_step": m["traversed_edges"],
                       "parallelism": f"replicas x{args.gpus}",
                       "l2": "256 MiB device write between timed steps (outside the events)"},
            "roofline": m["roofline"], "gpu_launches": m["gpu_launches"],
            "clocks": m["clocks"], "e2e": m.get("e2e"),
        }
        if "cpu_baseline" in m:
            line["cpu_baseline"] = m["cpu_baseline"]
        if extra:
            line["extra"] = extra
        print(json.dumps(line))
    dist.close()


if __name__ == "__main__":
    main()
