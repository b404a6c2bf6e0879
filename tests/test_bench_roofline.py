"""The roofline denominators bench.py reports: algorithmic bytes of a
work-optimal run, split into HBM and host-link bytes, on hand-counted toy
graphs (no GPU needed)."""
import importlib.util
import json
import os

import numpy as np
import pytest

ROOT = os.path.join(os.path.dirname(__file__), "..")


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


# 4 vertices, degrees 2, 1, 0, 2; blocks {0, 1} (resident) and {2, 3} (host)
OFF = np.array([0, 2, 3, 3, 5], np.uint64)
VB = np.array([0, 2, 4], np.uint32)
RES = np.array([True, False])


def test_traversal_bytes_split_by_residency(bench):
    vals = np.array([1, 2, 5, 3], np.uint32)  # vertex 2 unreached (n + 1)
    hbm, link, edges = bench.algorithmic_bytes(OFF, vals, 4, VB, RES, 4, "sssp")
    # reached: 0, 1 (resident, 3 edges) and 3 (host, 2 edges)
    assert link == 2 * 4
    assert hbm == 3 * 4 + 5 * 4 + 3 * (16 + 4)
    assert edges == 5


def test_small_list_cache_moves_short_host_lists_to_hbm(bench):
    vals = np.array([1, 2, 5, 3], np.uint32)
    hbm, link, _ = bench.algorithmic_bytes(OFF, vals, 4, VB, RES, 4, "bfs", list_deg=3)
    assert link == 0
    assert hbm == 5 * 4 + 5 * 4 + 3 * (16 + 4)


def test_whole_graph_algorithms_count_every_vertex_per_iteration(bench):
    vals = np.zeros(4, np.uint32)
    hbm, link, edges = bench.algorithmic_bytes(OFF, vals, 4, VB, RES, 4, "pr_push", n_iters=20)
    assert link == 20 * 2 * 4
    assert hbm == 20 * (3 * 4 + 5 * 8 + 4 * (16 + 4))
    assert edges == 5


def test_traffic_is_read_from_captures_of_the_same_workload(bench, tmp_path, monkeypatch):
    table = tmp_path / "t.json"
    table.write_text(json.dumps({"sssp_rmat24_wcsr_40%": {
        "dram_read_bytes": 1000, "dram_write_bytes": 24, "sysmem_read_sectors": 10,
        "command": "ncu ..."}}))
    monkeypatch.setattr(bench, "TRAFFIC_TABLE", str(table))
    dram, link, entry = bench.measured_traffic("sssp_rmat24_wcsr_40%")
    assert dram == 1024 and link == 320 and entry["command"] == "ncu ..."
    # a size that was not captured reports null, never a scaled guess
    assert bench.measured_traffic("sssp_rmat26_wcsr_40%") == (None, None, None)
    r = bench.roofline(100, 0, 1.0, 1.0, "measured", 1.0, 1.0, "sssp_rmat26_wcsr_40%", 1)
    assert r["traffic"] is None and r["link_traffic"] is None


def test_committed_traffic_table_entries_name_their_capture(bench):
    if not os.path.exists(bench.TRAFFIC_TABLE):
        pytest.skip("no captures committed")
    for key, e in json.load(open(bench.TRAFFIC_TABLE)).items():
        assert e["command"].startswith("ncu ") and "--clock-control none" in e["command"], key
        assert e["dram_read_bytes"] > 0, key


def test_union_find_bytes_skip_the_hub_component(bench):
    # degrees 3, 1, 4, 0, 3; the hub (vertex 2) shares label 0 with vertices
    # 0 and 1; vertices 3 and 4 are outside its component
    off = np.array([0, 3, 4, 8, 8, 11], np.uint64)
    labels = np.array([0, 0, 0, 3, 3], np.uint32)
    vb = np.array([0, 3, 5], np.uint32)
    res = np.array([True, False])
    hbm, link, edges = bench.algorithmic_bytes_cc_uf(off, labels, 5, vb, res, 4, 0)
    # sampled: min(deg, 2) = 2, 1, 2, 0, 2; the rest of a list only outside
    # the hub's component (vertex 4: one more edge; vertex 0 skips its third)
    assert edges == 2 + 1 + 2 + 0 + 3
    assert link == (0 + 3) * 4                     # vertices 3, 4 are on the host
    assert hbm == (2 + 1 + 2) * 4 + 8 * 8 + 5 * (16 + 12)
