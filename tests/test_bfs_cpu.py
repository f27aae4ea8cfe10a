"""The BFS oracle (bfs-rec's bfs_cpu restated, apps/bfs-rec/src/gpu/bfs_rec.cpp:100-119)
pinned to the reference's own bfs_cpu: against the golden levels it produced
(tests/golden/golden.json "bfs", written by tests/golden/make_golden.py) and,
where oracle/_ref/libref_bfs.so was built, against the reference run here."""
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
        want = golden["bfs"]["cases"][name]
        lv = oracle.bfs_levels(g.row_ptr, g.col, want["source"])
        assert lv.dtype == np.int32
        assert oracle.fnv1a(lv.view(np.uint32)) == want["levels_fnv1a"], name
        fin = lv[lv != oracle.BFS_UNDEFINED]
        assert fin.size == want["n_reached"] and int(fin.max()) == want["max_level"]


def test_oracle_edge_cases(nps, oracle, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        lv = oracle.bfs_levels(g.row_ptr, g.col, case["source"])
        assert lv.tolist() == golden["bfs"]["edge_cases"][name], name


def test_oracle_matches_reference_run_here(nps, oracle):
    if not oracle.have_reference_bfs():
        pytest.skip("oracle/_ref/libref_bfs.so not built (reference sources absent)")
    rng = np.random.default_rng(5)
    for g in (nps.gen_rmat(15, 8, seed=21), nps.gen_grid(90, 70, 0.1, 5, 4), nps.gen_uniform(20000, 60000, 9, 8)):
        for src in (g.source, int(rng.integers(0, g.n))):
            want, _ = oracle.ref_bfs_cpu(g.row_ptr, g.col, src)
            assert (oracle.bfs_levels(g.row_ptr, g.col, src) == want).all()


def test_bfs_arguments_are_checked(nps):
    g = nps.gen_uniform(100, 500, 10, 1)
    with pytest.raises(nps.NpsError) as ei:
        nps.bfs(g, g.n)  # source out of range
    assert ei.value.status == 1
    with pytest.raises(nps.NpsError) as ei:
        nps.bfs(g, 0, nps.bfs_params(block_size=96))
    assert ei.value.status == 1
