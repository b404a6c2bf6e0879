"""PageRank with the reference engine's own semantics.

tests/golden/ref_s14_pr_{pull,push}.f64 are results/values.bin of the
reference's GPU engine (tests/golden/make_ref_pr_golden.py) on the seeded
scale-14 graph; ref_pr_manifest.json records, for those runs and for scale-20
runs with all edges resident and with a 40% static budget, the largest
difference from the oracle's restatement (thvo_pagerank_ref_pull / _push).
The reference adds with FP64 atomics, so its sums are order-dependent and the
pin is its comparer's 1e-3 absolute tolerance (comparer/compare.cpp:155).
The engine's THV_RUN_PR_REFERENCE mode is held to the oracle much tighter.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MAN = json.load(open(os.path.join(GOLD, "ref_pr_manifest.json")))
TOL = MAN["tolerance_abs"]


def graph(O, name):
    p = MAN["graphs"][name]
    g = O.rmat(p["scale"], p["ef"], seed=MAN["seed"])
    assert (g.nv, g.ne) == (p["nv"], p["ne"])
    return g


def oracle_values(O, g, typ):
    if typ == "pull":
        return O.pagerank_ref_pull(*O.transpose(g))
    return O.pagerank_ref_push(g)


def test_reference_runs_agreed_with_the_oracle():
    # recorded on the B200, every run: resident and 40% budgets, scales 14 and 20
    assert {(r["graph"], r["type"], r["static_budget_frac"]) for r in MAN["runs"]} == {
        (n, t, f) for n in ("s14", "s20") for t in ("pull", "push") for f in (None, 0.4)}
    for r in MAN["runs"]:
        assert r["vertices_over_tolerance"] == 0 and r["max_abs_diff_vs_oracle"] <= TOL, r


@pytest.mark.parametrize("typ", ["pull", "push"])
def test_oracle_matches_reference_values(O, typ):
    g = graph(O, "s14")
    ref = np.fromfile(os.path.join(GOLD, f"ref_s14_pr_{typ}.f64"), np.float64)
    got, rounds = oracle_values(O, g, typ)
    assert rounds > 1
    assert ref.shape == got.shape
    assert np.abs(got - ref).max() <= TOL


def test_the_two_semantics_differ(O):
    # the reference's pull and push are different methods (un-normalised
    # Jacobi from 1/N, residual push from 0.15), and neither is the engine's
    # default fixed-iteration PageRank
    g = graph(O, "s14")
    pull, _ = oracle_values(O, g, "pull")
    push, _ = oracle_values(O, g, "push")
    fixed = O.pagerank(g)
    assert np.abs(pull - push).max() > 10 * TOL
    assert abs(pull.sum() - g.nv) > 1 and abs(fixed.sum() - 1.0) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("typ", ["pull", "push"])
@pytest.mark.parametrize("frac", [0.0, 0.4, 1.0])
def test_engine_reference_semantics_scale14(T, O, typ, frac):
    g = graph(O, "s14")
    ref = np.fromfile(os.path.join(GOLD, f"ref_s14_pr_{typ}.f64"), np.float64)
    want, rounds = oracle_values(O, g, typ)
    if typ == "pull":
        in_off, in_adj, outdeg = O.transpose(g)
        eg = T.Graph.from_arrays(in_off, in_adj, "csc", outdeg=outdeg)
    else:
        eg = T.Graph.from_arrays(g.off, g.adj, "csr")
    with eg:
        eg.plan(int(frac * eg.ne * 4), block_bytes=64 << 10)
        got, st = eg.run("pr_" + typ, pr_reference=True)
        assert st["iterations"] == rounds
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
        assert np.abs(got - ref).max() <= TOL
        # the fixed-iteration method still runs after it on the same graph
        fixed, _ = eg.run("pr_" + typ)
        np.testing.assert_allclose(fixed, O.pagerank(g), rtol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("typ", ["pull", "push"])
def test_engine_reference_semantics_scale20_split_tiles(T, O, typ):
    # scale 20: hubs are cut into several tiles (split vertices) and 60% of
    # the edges are read from host memory
    g = graph(O, "s20")
    want, rounds = oracle_values(O, g, typ)
    if typ == "pull":
        in_off, in_adj, outdeg = O.transpose(g)
        eg = T.Graph.from_arrays(in_off, in_adj, "csc", outdeg=outdeg)
    else:
        eg = T.Graph.from_arrays(g.off, g.adj, "csr")
    with eg:
        eg.plan(int(0.4 * eg.ne * 4), block_bytes=1 << 20)
        got, st = eg.run("pr_" + typ, pr_reference=True)
        assert st["iterations"] == rounds
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_engine_reference_semantics_round_cap(T, O):
    g = graph(O, "s14")
    with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
        eg.plan()
        with pytest.raises(T.ThvError) as e:
            eg.run("pr_push", pr_reference=True, pr_max_rounds=3)
        assert e.value.status == T.THV_ETIMEOUT
