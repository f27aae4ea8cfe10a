"""The SpMV oracle (spmv_omp restated, apps/SpMV/src/cpu/SpMV_kernel.cpp:26-42)
pinned to the reference's own SpMV_CPU path: against the golden y it produced
(tests/golden/golden.json "spmv", written by tests/golden/make_golden.py) and,
where oracle/_ref/libref_spmv.so was built, against the reference run here."""
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
    for name, case in golden["cases"].items():
        g = _gen(nps, case["kind"], case["args"])
        val, x = oracle.spmv_data(g.n, g.m)
        y = oracle.spmv(g.row_ptr, g.col, val, x)
        want = golden["spmv"]["cases"][name]
        assert oracle.fnv1a(y.view(np.uint32)) == want["y_fnv1a"], name
        assert float(y.sum()) == want["y_sum"] and float(y.max()) == want["y_max"]


def test_oracle_edge_cases(nps, oracle, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        val, x = oracle.spmv_data(g.n, g.m)
        assert oracle.spmv(g.row_ptr, g.col, val, x).tolist() == golden["spmv"]["edge_cases"][name], name


def test_oracle_matches_reference_run_here(nps, oracle):
    if not oracle.have_reference_spmv():
        pytest.skip("oracle/_ref/libref_spmv.so not built (reference sources absent)")
    for g in (nps.gen_rmat(15, 8, seed=21), nps.gen_grid(90, 70, 0.1, 5, 4), nps.gen_uniform(20000, 60000, 9, 8)):
        y, x, val, _ = oracle.ref_spmv_cpu(g.row_ptr, g.col, 4)
        v2, x2 = oracle.spmv_data(g.n, g.m)
        assert np.array_equal(val, v2) and np.array_equal(x, x2)
        assert np.array_equal(oracle.spmv(g.row_ptr, g.col, val, x), y)


def test_spmv_arguments_are_checked(nps):
    g = nps.gen_uniform(100, 500, 10, 1)
    with pytest.raises(ValueError):
        nps.spmv(g, np.ones(3), np.ones(g.n))


def test_spmv_levels_and_thresholds_are_checked_before_the_device(nps, oracle):
    g = nps.gen_uniform(100, 500, 10, 1)
    val, x = oracle.spmv_data(g.n, g.m)
    for kw in ({"level": 3}, {"level": -1}, {"threshold": 0}):
        with pytest.raises(nps.NpsError) as ei:
            nps.spmv(g, val, x, nps.Params(**kw))
        assert ei.value.status == 1, kw
