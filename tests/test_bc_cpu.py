"""The betweenness-centrality oracle (bc_cpu restated, apps/bc/src/cpu/bc.cpp:152-186
and bc_kernel.cpp:3-106) pinned to the reference's own bc_cpu: against the golden
centralities it produced (tests/golden/golden.json "bc", written by
tests/golden/make_golden.py) and, where oracle/_ref/libref_bc.so was built,
against the reference run here -- bit for bit, path-count wraparound included."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as f:
        return json.load(f)


def _gen(nps, kind, a):
    if kind == "uniform":
        return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])
    if kind == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])


def test_oracle_matches_reference_goldens(nps, oracle, golden):
    for name, case in golden["bc"]["cases"].items():
        g = _gen(nps, case["kind"], case["args"])
        b = oracle.bc(g.row_ptr, g.col)
        assert oracle.fnv1a(b.view(np.uint32)) == case["bc_fnv1a"], name
        assert float(b.max()) == case["bc_max"]


def test_oracle_edge_cases(nps, oracle, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        assert oracle.bc(g.row_ptr, g.col).tolist() == golden["bc"]["edge_cases"][name], name


def test_oracle_matches_reference_run_here(nps, oracle):
    if not oracle.have_reference_bc():
        pytest.skip("oracle/_ref/libref_bc.so not built (reference sources absent)")
    for g in (nps.gen_rmat(9, 16, seed=21), nps.gen_grid(20, 25, 0.2, 5, 4), nps.gen_uniform(700, 3000, 9, 8)):
        want, _ = oracle.ref_bc_cpu(g.row_ptr, g.col)
        assert np.array_equal(oracle.bc(g.row_ptr, g.col).view(np.uint32), want.view(np.uint32))


def test_source_subsets_fold_in_order(nps, oracle):
    """Sources given as a list are folded in list order: all sources in id order
    equal the default, and a prefix of them is a prefix of the fold."""
    g = nps.gen_rmat(9, 8, seed=2)
    full = oracle.bc(g.row_ptr, g.col)
    assert np.array_equal(oracle.bc(g.row_ptr, g.col, np.arange(g.n)), full)
    assert not np.array_equal(oracle.bc(g.row_ptr, g.col, np.arange(10)), full)


def test_bc_arguments_are_checked_before_the_device(nps):
    g = nps.gen_uniform(100, 500, 10, 1)
    for sources in ([0, 100], [-1], [5, 99, 1000]):
        with pytest.raises(nps.NpsError) as ei:
            nps.bc(g, sources)
        assert ei.value.status == 1, sources
