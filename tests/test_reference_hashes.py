"""Parity with the reference's own GPU engine at scales 20 and 22.

tests/golden/ref_hashes.json holds, per run, the sha256 of the
results/values.bin the reference's engine wrote on a B200
(tests/golden/make_ref_hashes.py; the build drops only the calls of the
diagnostic SetFrontierToRatio(), which zeroes the host frontier,
src/graph.cuh:160-163), next to the sha256 of the CPU oracle's answer.  The
runs with a static budget hold an HBM ballast, so the reference served the
rest of the edges through its demand kernels, and the scale-22 graphs span
several of its 64 MB partitions (src/bfs/bfs.cu:155-519, src/cc/cc.cu:71-614).

CPU tests regenerate each graph with the oracle's generator, check its hash,
and check the oracle's answer against the recorded hashes; GPU tests do the
same with the engine's generator and its BFS / CC at the same budgets.
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MAN = json.load(open(os.path.join(GOLD, "ref_hashes.json")))


def graph_sha(off, adj):
    """sha256 over off[0..nv) as u64 followed by the u32 adjacency."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(off[:-1], np.uint64).tobytes())
    h.update(np.ascontiguousarray(adj, np.uint32).tobytes())
    return h.hexdigest()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.uint32).tobytes()).hexdigest()


def runs_of(name):
    return [r for r in MAN["runs"] if r["graph"] == name]


def run_id(r):
    b = "full" if r["static_budget_frac"] is None else f"{int(r['static_budget_frac'] * 100)}pct"
    return f"{r['graph']}-{r['algo']}-src{r['source']}-{b}"


def test_reference_agreed_with_the_oracle_everywhere():
    # recorded on the B200: the reference's BFS and CC equal the oracle at
    # these sizes (its CC goes wrong only at scale 24 with a 40% budget)
    assert len(MAN["runs"]) == 9
    for r in MAN["runs"]:
        assert r["ref_equals_oracle"] and r["ref_sha256"] == r["oracle_sha256"], run_id(r)
    # the budgeted runs really left edges to the demand path
    for r in MAN["runs"]:
        if r["static_budget_frac"] is not None:
            assert r["static_edges"] < MAN["graphs"][r["graph"]]["ne"], run_id(r)


@pytest.mark.parametrize("name", sorted(MAN["graphs"]))
def test_oracle_reproduces_reference_hashes(O, name):
    p = MAN["graphs"][name]
    g = O.rmat(p["scale"], p["ef"], seed=MAN["seed"], symmetric=p["symmetric"])
    assert (g.nv, g.ne) == (p["nv"], p["ne"])
    assert graph_sha(g.off, g.adj) == p["graph_sha256"]
    for r in runs_of(name):
        got = O.bfs(g, r["source"], parallel=True) if r["algo"] == "bfs" else O.cc(g, parallel=True)
        assert sha(got) == r["ref_sha256"], run_id(r)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(MAN["graphs"]))
def test_engine_reproduces_reference_hashes(T, name):
    p = MAN["graphs"][name]
    with T.Graph.generate_rmat(p["scale"], p["ef"], seed=MAN["seed"], symmetric=p["symmetric"],
                               fmt="csr") as g:
        off, adj, _ = g.host_arrays()
        assert graph_sha(off, adj) == p["graph_sha256"]
        for r in runs_of(name):
            frac = r["static_budget_frac"]
            g.plan(None if frac is None else int(frac * g.ne * 4))
            got, _ = g.run(r["algo"], source=r["source"])
            assert sha(got) == r["ref_sha256"], run_id(r)
            if r["algo"] == "cc" and g.symmetric:
                # union-find is the default on symmetric graphs; the
                # reference's method must give the same labels
                got, _ = g.run("cc", label_propagation=True)
                assert sha(got) == r["ref_sha256"], run_id(r) + " label propagation"
