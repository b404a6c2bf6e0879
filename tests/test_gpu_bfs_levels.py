"""Direction-optimising BFS on graphs whose levels change size sharply.

Small top-down levels (at most 2,048 frontier vertices and out-edges) run
inside one CTA with block barriers and hand the frontier back to the grid
when a level grows; the grid's levels list the vertices they find when
they are small, so that the next level can go back to the CTA.  These
graphs walk that hand-over both ways, several times in one traversal:
- a long path (every level one vertex: the whole traversal in one CTA run);
- a path into a hub whose out-edges fan out to a large layer (the run must
  stop before the hub's level and the grid take it, top-down or
  bottom-up), the layer narrowing into another path (small levels again),
  then a second hub;
- an RMAT graph from sources whose first levels are tiny.
Every level is compared with the CPU oracle (levels are unique, so the
values are bit-exact whatever ran them).  Reference kernels replaced:
src/bfs/bfs_kernels.cu:4-76 and the level loop src/bfs/bfs.cu:55-524.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_bfs(T, g, src):
    with T.Graph.from_arrays(g.off, g.adj, "csr") as eg:
        eg.plan()  # every edge resident: the direction-optimising kernel
        got, st = eg.run("bfs", source=src)
    return got, st


def test_long_path_in_one_cta(T, O):
    n = 6000
    src = np.arange(n - 1, dtype=np.uint32)
    g = O.from_edges(n, src, src + 1)
    got, st = run_bfs(T, g, 0)
    assert np.array_equal(got, O.bfs(g, 0))
    assert got[n - 1] == n  # level n - 1, stored + 1
    assert st["iterations"] >= n - 1


def test_paths_and_hubs_hand_over_both_ways(T, O):
    rng = np.random.default_rng(5)
    srcs, dsts = [], []
    nxt = 0

    def path(length, start):
        nonlocal nxt
        ids = np.arange(nxt, nxt + length, dtype=np.int64)
        nxt += length
        srcs.extend([start] + list(ids[:-1]))
        dsts.extend(list(ids))
        return int(ids[-1])

    root = nxt
    nxt += 1
    end = path(40, root)
    for _ in range(2):
        hub = end
        layer = np.arange(nxt, nxt + 30000, dtype=np.int64)
        nxt += 30000
        srcs.extend([hub] * len(layer))
        dsts.extend(list(layer))
        # random edges inside the layer and back to it, so bottom-up levels
        # have parents to find
        a = rng.choice(layer, 60000)
        b = rng.choice(layer, 60000)
        srcs.extend(list(a))
        dsts.extend(list(b))
        end = path(50, int(layer[7]))
    n = nxt
    g = O.from_edges(n, np.array(srcs, np.uint32), np.array(dsts, np.uint32))
    got, _ = run_bfs(T, g, root)
    assert np.array_equal(got, O.bfs(g, root))


def test_rmat_tiny_first_levels(T, O):
    g = O.rmat(16, 16)
    deg = np.diff(g.off.astype(np.int64))
    # low-degree sources: the first levels are tiny and run in one CTA
    cand = np.flatnonzero((deg > 0) & (deg <= 2))[:6]
    for s in cand:
        got, _ = run_bfs(T, g, int(s))
        assert np.array_equal(got, O.bfs(g, int(s))), int(s)
