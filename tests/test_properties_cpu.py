"""Properties the oracles of the widened paths must have, independent of the
reference runs that pin them: BFS levels are unit-weight shortest paths, colors
increase along every edge to a smaller vertex, y = A x is linear, and
betweenness on a directed path has its closed form."""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_bfs_levels_are_unit_weight_distances(nps, oracle, seed):
    for g in (nps.gen_rmat(12, 8, seed=seed), nps.gen_uniform(3000, 12000, 9, seed), nps.gen_grid(30, 40, 0.1, 9, seed)):
        lv = oracle.bfs_levels(g.row_ptr, g.col, g.source)
        d = oracle.sssp_heap(g.row_ptr, g.col, np.ones(g.m, np.uint32), g.source)
        reached = d < oracle.INF
        assert np.array_equal(reached, lv != oracle.BFS_UNDEFINED)
        assert np.array_equal(lv[reached].astype(np.uint32), d[reached])


@pytest.mark.parametrize("seed", [1, 2])
def test_colors_increase_towards_larger_vertices(nps, oracle, seed):
    g = nps.gen_rmat(13, 8, seed=seed)
    c, it = oracle.color(g.row_ptr, g.col)
    src = np.repeat(np.arange(g.n), np.diff(g.row_ptr))
    smaller = g.col < src
    assert np.all(c[src[smaller]] > c[g.col[smaller]])  # no edge to a smaller vertex shares a color
    assert c.min() == 1 and it == c.max()


def test_spmv_is_linear(nps, oracle):
    g = nps.gen_rmat(12, 8, seed=4)
    rng = np.random.default_rng(0)
    val = rng.integers(-8, 9, g.m).astype(np.float64)  # small integers: every sum is exact
    x1 = rng.integers(-8, 9, g.n).astype(np.float64)
    x2 = rng.integers(-8, 9, g.n).astype(np.float64)
    y = oracle.spmv(g.row_ptr, g.col, val, x1 + 3 * x2)
    assert np.array_equal(y, oracle.spmv(g.row_ptr, g.col, val, x1) + 3 * oracle.spmv(g.row_ptr, g.col, val, x2))


@pytest.mark.parametrize("k", [2, 5, 17])
def test_bc_on_a_directed_path(nps, oracle, k):
    """0 -> 1 -> ... -> k-1: vertex i lies on the single shortest path of every pair
    s < i < t, so bc(i) = i * (k - 1 - i)."""
    g = nps.convertCSR(k, np.arange(k - 1), np.arange(1, k), np.ones(k - 1, np.uint32))
    b = oracle.bc(g.row_ptr, g.col)
    assert b.tolist() == [float(i * (k - 1 - i)) for i in range(k)]
