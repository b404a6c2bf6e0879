"""Hashes of the reference GPU engine's BFS / CC output at scales 20 and 22.

Runs oracle/_ref/thv_ref (the reference's src/ compiled for sm_100a by
oracle/Makefile, with only the calls of its diagnostic SetFrontierToRatio()
dropped: that function zeroes the host frontier, src/graph.cuh:160-163) on
seeded RMAT graphs written in the converter's .csr format, and records the
sha256 of each results/values.bin next to the sha256 of the CPU oracle's
answer.  The runs with a static budget hold an HBM ballast (the wrapper's
--static-budget), so the reference serves the rest of the edges through its
demand (zero-copy) kernels; the scale-22 graphs span 4 (directed) and 8
(symmetric) of its 64 MB partitions, so its partition-cost and filter code
runs as well (src/bfs/bfs.cu:155-519, src/cc/cc.cu:71-614).

The values are 4 MB to 16 MB each, so only their hashes are committed
(tests/golden/ref_hashes.json); tests regenerate the graphs, check the
graph hash, and compare the hash of their own output.  Needs a GPU; the
output directory is argv[1] (default: this directory).
"""
import hashlib
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
GRAPHS = {
    "s20": dict(scale=20, ef=16, symmetric=False),
    "s20sym": dict(scale=20, ef=16, symmetric=True),
    "s22": dict(scale=22, ef=16, symmetric=False),
    "s22sym": dict(scale=22, ef=16, symmetric=True),
}
# (graph, algo, source, static budget as a fraction of the edge bytes or None)
RUNS = [
    ("s20", "bfs", 1, None),
    ("s20", "bfs", 1, 0.4),
    ("s20", "bfs", "seeded0", 0.4),
    ("s20", "bfs", "seeded1", 0.4),
    ("s22", "bfs", 1, 0.4),
    ("s20", "cc", 0, 0.4),
    ("s20sym", "cc", 0, None),
    ("s20sym", "cc", 0, 0.4),
    ("s22sym", "cc", 0, 0.4),
]


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def graph_sha(off: np.ndarray, adj: np.ndarray) -> str:
    """sha256 over off[0..nv) as u64 followed by the u32 adjacency."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off[:-1], np.uint64).tobytes())
    h.update(np.ascontiguousarray(adj, np.uint32).tobytes())
    return h.hexdigest()


def graph(name):
    p = GRAPHS[name]
    return O.rmat(p["scale"], p["ef"], symmetric=p["symmetric"])


def resolve_source(g, src):
    if isinstance(src, str):
        return int(O.sources(g, int(src[len("seeded"):]) + 1)[-1])
    return int(src)


def main(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    man = {"seed": O.SEED, "graphs": {}, "runs": []}
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "results"))
    try:
        for name in GRAPHS:
            runs = [r for r in RUNS if r[0] == name]
            if not runs:
                continue
            g = graph(name)
            path = os.path.join(work, f"{name}.csr")
            O.write_csr(path, g)
            man["graphs"][name] = dict(GRAPHS[name], nv=g.nv, ne=g.ne,
                                       graph_sha256=graph_sha(g.off, g.adj))
            for _, algo, src_spec, frac in runs:
                src = resolve_source(g, src_spec) if algo == "bfs" else 0
                cmd = [REF, "--input", path, "--algo", algo, "--source", str(src), "--runs", "1"]
                if frac is not None:
                    cmd += ["--static-budget", str(int(frac * g.ne * 4))]
                vb = os.path.join(work, "results", "values.bin")
                if os.path.exists(vb):
                    os.unlink(vb)
                r = subprocess.run(cmd, cwd=work, capture_output=True, text=True, timeout=600)
                if r.returncode != 0:
                    raise RuntimeError(f"reference {algo} on {name} failed: {r.stdout[-800:]} {r.stderr[-800:]}")
                vals = np.fromfile(vb, np.uint32)
                want = O.bfs(g, src, parallel=True) if algo == "bfs" else O.cc(g, parallel=True)
                rec = {"graph": name, "algo": algo, "source": src, "source_spec": src_spec,
                       "static_budget_frac": frac,
                       "static_edges": next((int(ln.split(":")[1]) for ln in r.stdout.splitlines()
                                             if ln.startswith("Number of static edges")), None),
                       "ref_sha256": sha(vals.tobytes()), "oracle_sha256": sha(want.tobytes()),
                       "ref_equals_oracle": bool(np.array_equal(vals, want)),
                       "reached_or_labels": int((want < g.nv + 1).sum()) if algo == "bfs"
                       else int(len(np.unique(want))),
                       "reference_log": next((ln for ln in r.stdout.splitlines()
                                              if "Average execution time" in ln), "")}
                if not rec["ref_equals_oracle"]:
                    rec["mismatch_vertices"] = int((vals != want).sum())
                    rec["ref_above_oracle"] = int((vals > want).sum())
                man["runs"].append(rec)
                print(json.dumps(rec), flush=True)
            os.unlink(path)
        json.dump(man, open(os.path.join(out_dir, "ref_hashes.json"), "w"), indent=1)
    finally:
        shutil.rmtree(work)
    print("wrote", os.path.join(out_dir, "ref_hashes.json"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
