"""Time the reference's own GPU engine (oracle/_ref/thv_ref) on the configs.

Test/measurement infrastructure: generates each graph with the CPU oracle,
writes it in the converter's format (.csr, or .csc for pull PageRank), runs
the reference with --runs N (HBM budgets forced with the wrapper's ballast,
since the reference sizes its static region from free memory itself,
src/graph.cuh:306-341), parses its "Average execution time", samples the SM
clocks while it runs, and checks BFS/CC values against the oracle.

GTEPS uses the engine's definitions: BFS/SSSP count the out-degrees of the
reached vertices, CC all edges.  The reference's PageRank runs until every
vertex changes by at most 1e-3 (src/pr/pr_kernels.cu:449-476, :846-860), not
for a fixed iteration count, and its values follow other semantics (FP64,
un-normalised, no dangling redistribution), so for PageRank only the time
per run is comparable; its values are recorded by hash only.

Prints one JSON object per case.  Needs a GPU.

  python oracle/ref_gpu_timing.py [case ...]     (default: every case)
"""
import hashlib
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle import oracle as O  # noqa: E402

PR_BUDGET = 2 << 30  # config 3: 2 GiB of HBM for edges

CASES = {
    "c1_bfs": dict(scale=20, ef=16, sym=False, algo="bfs", src=1, budget=None, runs=5),
    "c2_cc": dict(scale=24, ef=16, sym=True, algo="cc", src=0, frac=0.4, runs=5),
    "c2_sssp": dict(scale=24, ef=16, sym=False, algo="sssp", src=1, frac=0.4, runs=5),
    "c3_pr_pull": dict(scale=26, ef=16, sym=False, algo="pr", type="pull", src=0,
                       budget=PR_BUDGET, runs=2, timeout=900),
    "c3_pr_push": dict(scale=26, ef=16, sym=False, algo="pr", type="push", src=0,
                       budget=PR_BUDGET, runs=2, timeout=900),
}

CLOCK_Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
           "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
           "clocks_event_reasons.sw_power_cap")


def is_fixed_point(g, lab):
    """True if no edge u->w has lab[u] < lab[w] (propagation converged)."""
    deg = np.diff(g.off.astype(np.int64))
    src = np.repeat(np.arange(g.nv), deg)
    return not np.any(lab[src] < lab[g.adj])


def sha(b):
    return hashlib.sha256(b).hexdigest()


class Clocks:
    """nvidia-smi samples every 200 ms while the reference runs."""

    def __init__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.p = subprocess.Popen(["nvidia-smi", "-i", "0", f"--query-gpu={CLOCK_Q}",
                                   "--format=csv,noheader,nounits", "-lms", "200"],
                                  stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self):
        self.p.terminate()
        self.p.wait(timeout=10)
        rows = [[x.strip() for x in ln.split(",")] for ln in open(self.path)]
        os.unlink(self.path)
        rows = [r for r in rows if len(r) >= 7]
        busy = [float(r[0]) for r in rows if float(r[2]) > 250] or [float(r[0]) for r in rows] or [0]
        reasons = [n for i, n in [(3, "hw_slowdown"), (4, "hw_thermal_slowdown"),
                                  (5, "sw_thermal_slowdown"), (6, "sw_power_cap")]
                   if any(r[i].lower().startswith("active") for r in rows)]
        return {"sm_mhz_median_busy": statistics.median(busy),
                "sm_max_mhz": max([float(r[1]) for r in rows] or [0]),
                "reasons": reasons, "samples": len(rows)}


def main(names):
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "results"))
    try:
        for name in names:
            run_case(name, CASES[name], work)
    finally:
        shutil.rmtree(work)


def run_case(name, c, work):
    t0 = time.time()
    g = O.rmat(c["scale"], c["ef"], symmetric=c["sym"])
    pull = c["algo"] == "pr" and c.get("type") == "pull"
    path = os.path.join(work, f"{name}.{'csc' if pull else 'csr'}")
    (O.write_csc if pull else O.write_csr)(path, g)
    gen_s = time.time() - t0
    exe = os.path.join(HERE, "_ref", "thv_ref")
    cmd = [exe, "--input", path, "--algo", c["algo"], "--source", str(c["src"]),
           "--runs", str(c["runs"])]
    if c["algo"] == "pr":
        cmd += ["--type", c["type"]]
    budget = c.get("budget")
    if "frac" in c:
        budget = int(c["frac"] * g.ne * 4)
    if budget is not None:
        cmd += ["--static-budget", str(budget)]
    vb = os.path.join(work, "results", "values.bin")
    if os.path.exists(vb):
        os.unlink(vb)
    ck = Clocks()
    try:
        r = subprocess.run(cmd, cwd=work, capture_output=True, text=True,
                           timeout=c.get("timeout", 600))
    except subprocess.TimeoutExpired as e:
        r = subprocess.CompletedProcess(cmd, "timeout", e.stdout or "", e.stderr or "")
        if isinstance(r.stdout, bytes):
            r.stdout, r.stderr = r.stdout.decode(errors="replace"), (r.stderr or b"").decode(errors="replace")
    clocks = ck.stop()
    os.unlink(path)
    m = re.findall(r"Average execution time: ([0-9.eE+-]+) ms", r.stdout)
    runs = [float(x) for x in re.findall(r"Execution time: :? *([0-9.eE+-]+) ms", r.stdout)]
    st = re.findall(r"Number of static edges: (\d+)", r.stdout)
    res = {"case": name,
           "cmd": " ".join(["oracle/_ref/thv_ref", "--input", os.path.basename(path)] + cmd[3:]),
           "rc": r.returncode, "avg_ms": float(m[-1]) if m else None, "run_ms": runs,
           "static_edges": int(st[-1]) if st else None, "nv": g.nv, "ne": g.ne,
           "static_budget_bytes": budget, "clocks": clocks, "graph_build_s": round(gen_s, 1)}
    raw = open(vb, "rb").read() if os.path.exists(vb) else b""
    res["values_sha256"] = sha(raw) if raw else None
    if c["algo"] in ("bfs", "cc", "sssp"):
        vals = np.frombuffer(raw, np.uint32) if raw else np.zeros(0, np.uint32)
        if c["algo"] == "bfs":
            want = O.bfs(g, c["src"], parallel=True)
            res["traversed"] = O.reached_edges(g, want)
        elif c["algo"] == "cc":
            want = O.cc(g, parallel=True)
            res["traversed"] = g.ne
        else:
            gw = O.CSR(g.off, g.adj, O.weights(g))
            want = O.sssp(gw, c["src"], parallel=True)
            res["traversed"] = O.reached_edges(g, want)
            res["note"] = "reference SSSP ignores the file weights (defect F1)"
        res["oracle_sha256"] = sha(want.tobytes())
        res["bit_exact_vs_oracle"] = bool(len(vals) == g.nv and np.array_equal(vals, want))
        if len(vals) == g.nv and not res["bit_exact_vs_oracle"]:
            res["mismatch"] = {"vertices": int((vals != want).sum()),
                               "ref_above_oracle": int((vals > want).sum()),
                               "ref_below_oracle": int((vals < want).sum()),
                               "ref_distinct": int(len(np.unique(vals))),
                               "oracle_distinct": int(len(np.unique(want)))}
            if c["algo"] == "cc":
                res["mismatch"]["ref_is_fixed_point"] = bool(is_fixed_point(g, vals))
        if res["avg_ms"]:
            res["gteps"] = res["traversed"] / (res["avg_ms"] * 1e-3) / 1e9
    else:
        res["note"] = ("reference PageRank: FP64, runs until every vertex changes by <= 1e-3, "
                       "un-normalised, no dangling redistribution; time per converged run only")
        if raw:
            v = np.frombuffer(raw, np.float64)
            res["ref_value_stats"] = {"min": float(v.min()), "max": float(v.max()),
                                      "sum": float(v.sum())}
    res["log_tail"] = r.stdout[-400:] + r.stderr[-400:]
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
