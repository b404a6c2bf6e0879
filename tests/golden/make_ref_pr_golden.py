"""Golden PageRank vectors from the reference's own GPU engine.

The reference's PageRank is tolerance-driven FP64 (src/common.cuh:48-49,
src/pr/pr_kernels.cu:449-476 pull, :846-860 push), another method than the
engine's default fixed-iteration FP32 PageRank; the engine reproduces it
under THV_RUN_PR_REFERENCE, and the oracle restates it
(thvo_pagerank_ref_pull / _push).  This script runs oracle/_ref/thv_ref --
the reference's src/ built by oracle/Makefile -- with --algo pr --type pull
on a .csc and --type push on a .csr, stores results/values.bin (nv doubles)
of the full-budget scale-14 runs, and records for every run (scale 14 and
scale 20; all edges resident, and a 40% static budget that leaves the rest
to the reference's demand kernels) the largest absolute difference from the
oracle.  Its FP64 atomics make the reference's sums order-dependent, so the
comparison is within the reference comparer's own 1e-3 absolute tolerance
(comparer/compare.cpp:155), not bitwise.  Needs a GPU; writes into argv[1]
(default: this directory).
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "thv_ref")
GRAPHS = {"s14": dict(scale=14, ef=8), "s20": dict(scale=20, ef=16)}


def run_ref(path, typ, work, budget=None):
    res = os.path.join(work, "results")
    os.makedirs(res, exist_ok=True)
    vb = os.path.join(res, "values.bin")
    if os.path.exists(vb):
        os.unlink(vb)
    cmd = [REF, "--input", path, "--algo", "pr", "--type", typ, "--runs", "1"]
    if budget is not None:
        cmd += ["--static-budget", str(budget)]
    r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"reference pr {typ} failed: {r.stdout[-1000:]} {r.stderr[-1000:]}")
    return np.fromfile(vb, np.float64), r.stdout


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    man = {"seed": O.SEED, "tolerance_abs": 1e-3, "graphs": {}, "runs": []}
    work = tempfile.mkdtemp()
    try:
        for name, p in GRAPHS.items():
            g = O.rmat(p["scale"], p["ef"])
            csr = os.path.join(work, f"{name}.csr")
            csc = os.path.join(work, f"{name}.csc")
            O.write_csr(csr, g)
            O.write_csc(csc, g)
            in_off, in_adj, outdeg = O.transpose(g)
            want = {"pull": O.pagerank_ref_pull(in_off, in_adj, outdeg),
                    "push": O.pagerank_ref_push(g)}
            man["graphs"][name] = dict(p, nv=g.nv, ne=g.ne)
            for typ, path in (("pull", csc), ("push", csr)):
                for frac in (None, 0.4):
                    budget = None if frac is None else int(frac * g.ne * 4)
                    got, log = run_ref(path, typ, work, budget)
                    ov, rounds = want[typ]
                    assert got.shape == ov.shape, (name, typ, got.shape)
                    diff = np.abs(got - ov)
                    fn = None
                    if name == "s14" and frac is None:
                        fn = f"ref_s14_pr_{typ}.f64"
                        got.tofile(os.path.join(out_dir, fn))
                    t = [ln for ln in log.splitlines() if "Average execution time" in ln]
                    man["runs"].append({
                        "graph": name, "type": typ, "static_budget_frac": frac, "file": fn,
                        "oracle_rounds": rounds, "max_abs_diff_vs_oracle": float(diff.max()),
                        "vertices_over_tolerance": int((diff > 1e-3).sum()),
                        "max_rel_diff_vs_oracle": float((diff / np.maximum(np.abs(ov), 1e-300)).max()),
                        "reference_log": t[-1] if t else ""})
                    print(json.dumps(man["runs"][-1]), flush=True)
        json.dump(man, open(os.path.join(out_dir, "ref_pr_manifest.json"), "w"), indent=1)
    finally:
        shutil.rmtree(work)
    print("wrote", out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
