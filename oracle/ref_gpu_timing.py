"""Time the reference's own GPU engine (oracle/_ref/thv_ref) on the configs.

Test/measurement infrastructure: generates each graph with the CPU oracle,
writes it in the converter's .csr format, runs the reference with --runs N
(HBM budgets forced with the wrapper's ballast), parses its "Average
execution time", and checks BFS/CC values against the oracle.  GTEPS uses
the engine's definitions (BFS/SSSP: out-degrees of reached vertices; CC:
all edges).  Prints one JSON object per case.  Needs a GPU.
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle import oracle as O  # noqa: E402

CASES = {
    "c1_bfs": dict(scale=20, ef=16, sym=False, algo="bfs", src=1, frac=None),
    "c2_cc": dict(scale=24, ef=16, sym=True, algo="cc", src=0, frac=0.4),
    "c2_sssp": dict(scale=24, ef=16, sym=False, algo="sssp", src=1, frac=0.4),
}


def is_fixed_point(g, lab):
    """True if no edge u->w has lab[u] < lab[w] (propagation converged)."""
    deg = np.diff(g.off.astype(np.int64))
    src = np.repeat(np.arange(g.nv), deg)
    return not np.any(lab[src] < lab[g.adj])


def main(names, runs=5):
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "results"))
    for name in names:
        c = CASES[name]
        g = O.rmat(c["scale"], c["ef"], symmetric=c["sym"])
        path = os.path.join(work, f"{name}.csr")
        O.write_csr(path, g)
        cmd = [os.path.join(HERE, "_ref", "thv_ref"), "--input", path, "--algo", c["algo"],
               "--source", str(c["src"]), "--runs", str(runs)]
        if c["frac"] is not None:
            cmd += ["--static-budget", str(int(c["frac"] * g.ne * 4))]
        r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=1800)
        m = re.findall(r"Average execution time: ([0-9.eE+-]+) ms", r.stdout)
        st = re.findall(r"Number of static edges: (\d+)", r.stdout)
        vals = np.fromfile(os.path.join(work, "results", "values.bin"), np.uint32)
        res = {"case": name, "rc": r.returncode, "avg_ms": float(m[-1]) if m else None,
               "static_edges": int(st[-1]) if st else None, "ne": g.ne}
        if c["algo"] == "bfs":
            want = O.bfs(g, c["src"], parallel=True)
            res["traversed"] = O.reached_edges(g, want)
            res["bit_exact_vs_oracle"] = bool(np.array_equal(vals, want))
        elif c["algo"] == "cc":
            res["traversed"] = g.ne
            want = O.cc(g, parallel=True)
            res["bit_exact_vs_oracle"] = bool(np.array_equal(vals, want))
            diff = vals != want
            res["mismatch"] = {"vertices": int(diff.sum()),
                               "ref_above_oracle": int((vals > want).sum()),
                               "ref_below_oracle": int((vals < want).sum()),
                               "ref_labels": int(len(np.unique(vals))),
                               "oracle_labels": int(len(np.unique(want))),
                               "ref_is_fixed_point": bool(is_fixed_point(g, vals))}
        else:
            gw = O.CSR(g.off, g.adj, O.weights(g))
            want = O.sssp(gw, c["src"], parallel=True)
            res["traversed"] = O.reached_edges(g, want)
            res["bit_exact_vs_oracle"] = bool(np.array_equal(vals, want))
            res["note"] = "reference SSSP ignores the file weights (defect F1)"
        if res["avg_ms"]:
            res["gteps"] = res["traversed"] / (res["avg_ms"] * 1e-3) / 1e9
        res["log_tail"] = r.stdout[-600:]
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
