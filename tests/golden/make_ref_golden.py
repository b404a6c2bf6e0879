"""Golden BFS / CC vectors from the reference's own GPU engine.

Runs oracle/_ref/thv_ref -- the reference's src/ compiled for sm_100a by
oracle/Makefile with one patch: the calls of its diagnostic
SetFrontierToRatio() are dropped, because that function zeroes the host
frontier (src/graph.cuh:160-163) so the unmodified engine never traverses
-- on seeded RMAT graphs written in the converter's .csr format, and stores
results/values.bin of each run.  The unmodified build (oracle/_ref/
thv_ref_asis) is run once per algorithm too and its output recorded, to
show it returns the initial values.  Needs a GPU; writes into the directory
given as argv[1] (default: this directory).

Graphs (oracle generator, seed 0x54484592): directed scale 14 / edge factor
8, and its symmetric counterpart (scale 14 / edge factor 4).  Both have more
than 14000 vertices so the reference's SetFrontierToRatio loop bound
(src/graph.cuh:182) does not underflow.  BFS and CC are deterministic fixed
points (min-relaxation), so the reference's output is exact.
"""
import hashlib
import json

import numpy as np
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "thv_ref")
REF_ASIS = os.path.join(ROOT, "oracle", "_ref", "thv_ref_asis")
GRAPHS = {"s14": dict(scale=14, ef=8, symmetric=False), "s14sym": dict(scale=14, ef=4, symmetric=True)}


def graph(name):
    p = GRAPHS[name]
    return O.rmat(p["scale"], p["ef"], symmetric=p["symmetric"])


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def run_ref(path, algo, src, work, exe=REF):
    res = os.path.join(work, "results")
    os.makedirs(res, exist_ok=True)
    vb = os.path.join(res, "values.bin")
    if os.path.exists(vb):
        os.unlink(vb)
    r = subprocess.run([exe, "--input", path, "--algo", algo, "--source", str(src), "--runs", "1"],
                       cwd=work, capture_output=True, text=True, timeout=300)
    if r.returncode != 0:
        raise RuntimeError(f"reference {algo} failed: {r.stderr[-2000:]}")
    return open(vb, "rb").read(), r.stdout


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    manifest = {"seed": O.SEED, "graphs": {}, "runs": []}
    work = tempfile.mkdtemp()
    try:
        for name in GRAPHS:
            g = graph(name)
            path = os.path.join(work, f"{name}.csr")
            O.write_csr(path, g)
            manifest["graphs"][name] = dict(GRAPHS[name], nv=g.nv, ne=g.ne, csr_sha256=sha(path))
            jobs = [("cc", 0)]
            if name == "s14":
                jobs += [("bfs", int(s)) for s in [1] + O.sources(g, 3).tolist()]
            for algo, src in jobs:
                vals, log = run_ref(path, algo, src, work)
                fn = f"ref_{name}_{algo}" + (f"_src{src}" if algo == "bfs" else "") + ".u32"
                open(os.path.join(out_dir, fn), "wb").write(vals)
                t = [ln for ln in log.splitlines() if "Average execution time" in ln]
                manifest["runs"].append({"graph": name, "algo": algo, "source": src, "file": fn,
                                         "reference_log": t[-1] if t else ""})
        # the unmodified build: does it traverse at all?
        g = graph("s14")
        path = os.path.join(work, "s14.csr")
        asis = {}
        s0 = int(O.sources(g, 1)[0])
        for algo, src, want in [("bfs", s0, O.bfs(g, s0)), ("cc", 0, O.cc(g))]:
            vals, _ = run_ref(path, algo, src, work, exe=REF_ASIS)
            v = np.frombuffer(vals, np.uint32)
            init = np.arange(g.nv, dtype=np.uint32) if algo == "cc" else np.where(
                np.arange(g.nv) == src, 1, g.nv + 1).astype(np.uint32)
            asis[algo] = {"equals_initial_values": bool(np.array_equal(v, init)),
                          "equals_oracle": bool(np.array_equal(v, want))}
        manifest["unmodified_reference"] = asis
        json.dump(manifest, open(os.path.join(out_dir, "ref_manifest.json"), "w"), indent=1)
    finally:
        shutil.rmtree(work)
    print("wrote", out_dir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
