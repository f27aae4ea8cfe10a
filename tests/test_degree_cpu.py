"""The degree-statistics oracle (oracle.degree_stats, a restatement of the
reference analyzer's getStatInfo(), utility/graph-analyzer/analyzer.cpp:75-138)
against the golden outputs of the reference analyzer itself."""
import importlib
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))["analyzer"]
READERS = {0: "readInputDIMACS9", 1: "readInputDIMACS10", 2: "readInputSLNDC"}


def graph_of(nps, name, rec):
    if "file" in rec:
        return getattr(nps, READERS[rec["format"]])(os.path.join(HERE, "golden", rec["file"]))
    a = rec["args"]
    if rec["kind"] == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    if rec["kind"] == "uniform":
        return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])
    return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])


def matches_golden(st, rec):
    for k in ("n", "m", "edges_by_degree", "max_degree", "min_degree", "max_degree_node", "min_degree_node"):
        assert st[k] == rec[k], k
    assert st["avg_degree"] == pytest.approx(rec["avg_degree"], abs=5e-7, rel=1e-6)  # printed with %f
    dist = [[i, int(c)] for i, c in enumerate(np.asarray(st["dist"])) if c]
    assert dist == rec["dist"]


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_matches_the_reference_analyzer(nps, oracle, name):
    rec = GOLD[name]
    g = graph_of(nps, name, rec)
    matches_golden(oracle.degree_stats(g.row_ptr), rec)


def test_oracle_edge_cases(oracle):
    st = oracle.degree_stats(np.array([0, 0, 0], np.int32))  # two isolated vertices
    assert (st["max_degree"], st["min_degree"], st["max_degree_node"], st["min_degree_node"]) == (0, 0, 0, 0)
    st = oracle.degree_stats(np.array([0, 3, 3, 5], np.int32))
    assert st["bins"] == [2, 1, 0, 0, 0, 0, 0, 0]  # degrees 3, 0, 2: bins [0, 3), [3, 15)
    assert st["max_degree_node"] == 0 and st["min_degree_node"] == 1 and list(st["dist"]) == [1, 0, 1, 1]
