"""The graph-coloring oracle, pinned to the reference's own program.

tests/golden/color_reference.json holds the colors that the reference's
gpu-graph-color (apps/graph-color/src/gpu, built from its sources by
oracle/Makefile; `-s 0`: gclr_nopruning_gpu(), one gclr_bitmap_kernel launch per
color, graph_color_kernel.cu:14-35) computed on a B200 for the three golden
reader files and four generated graphs (tests/golden/make_color_golden.py).  The
oracle's closed form, color(v) = 1 + the largest color of v's smaller
out-neighbours, must equal them; it must also equal a literal simulation of the
reference's iterations (every iteration tests every uncolored vertex against the
colors of the moment, including ones colored earlier in the same iteration)."""
import json
import os

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


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _fnv1a(a):
    h = 1469598103934665603
    for x in np.asarray(a, dtype=np.uint32).tolist():
        h = ((h ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_closed_form_equals_the_reference_program(nps, oracle):
    with open(os.path.join(GOLDEN, "color_reference.json")) as f:
        ref = json.load(f)["graphs"]
    readers = {0: nps.readInputDIMACS9, 1: nps.readInputDIMACS10, 2: nps.readInputSLNDC}
    for name, r in ref.items():
        if "colors" in r:  # a golden reader file
            g = readers[r["format"]](os.path.join(GOLDEN, name))
            c, it = oracle.color(g.row_ptr, g.col)
            assert c.tolist() == r["colors"], name
        else:  # a generated graph, written as DIMACS9 and read back by the reference
            g = getattr(nps, r["generator"])(**r["args"])
            c, it = oracle.color(g.row_ptr, g.col)
            assert str(_fnv1a(c)) == r["fnv1a"], name
        assert c.size == r["n"] and it == r["max_color"], name
