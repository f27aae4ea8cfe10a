"""The graph-coloring oracle.  The reference has no CPU version of graph-color
and its GPU code is not run here, so parity is unpinned: the oracle restates the
kernel (gclr_bitmap_kernel, apps/graph-color/src/gpu/graph_color_kernel.cu:14-35)
twice and the two must agree -- a literal simulation of the reference's
iterations (every iteration tests every uncolored vertex against the colors of
the moment, including ones colored earlier in the same iteration) and the
closed form the GPU computes, color(v) = 1 + the largest color of v's smaller
out-neighbours."""
import numpy as np
import pytest


@pytest.mark.parametrize("kind", ["rmat", "grid", "uniform", "edge"])
def test_closed_form_equals_the_literal_iterations(nps, oracle, kind):
    gs = {"rmat": [nps.gen_rmat(12, 16, seed=3), nps.gen_rmat(10, 4, seed=8)],
          "grid": [nps.gen_grid(40, 40, 0.1, 10, 1), nps.gen_grid(13, 70, 0.0, 10, 2)],
          "uniform": [nps.gen_uniform(3000, 20000, 10, 2)],
          "edge": [nps.convertCSR(5, [1, 2, 0, 0, 4], [2, 3, 1, 1, 0], [4, 5, 1, 1, 1]),
                   nps.convertCSR(1, [], [], []), nps.convertCSR(4, [3, 3, 3, 2], [3, 2, 1, 0], [1, 1, 1, 1])]}[kind]
    for g in gs:
        a, ia = oracle.color(g.row_ptr, g.col)
        b, ib = oracle.color(g.row_ptr, g.col, literal=True)
        assert np.array_equal(a, b) and ia == ib
        assert a.min() >= 1 and ia == a.max()


def test_color_arguments_are_checked(nps):
    g = nps.gen_uniform(100, 500, 10, 1)
    with pytest.raises(nps.NpsError) as ei:
        nps.color(g, nps.Params(threshold=0))
    assert ei.value.status == 1
