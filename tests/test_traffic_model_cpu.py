"""The host-side byte model used by the profiles (nested-parallelism_b200/traffic_model.py):
on a small R-MAT graph its reached set equals the CPU oracle's, and its sector counts bound
the useful bytes from above and add up over the degree classes."""
import importlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "nested-parallelism_b200"))


def test_model_on_rmat14(nps, oracle):
    tm = importlib.import_module("traffic_model")
    g = nps.gen_rmat(14, 16, seed=5)
    row, col = np.asarray(g.row_ptr), np.asarray(g.col)
    t = tm.model(row, col, g.source)
    d = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    r = d < oracle.INF
    assert t["n_r"] == int(r.sum())
    assert t["m_r"] == int(np.diff(row.astype(np.int64))[r].sum())
    assert t["b_alg"] == 12 * t["m_r"] + 12 * t["n_r"] + 4 * t["n"]
    assert t["csr_sectors"] >= t["csr_useful"] and t["row_ptr_sectors"] >= t["row_ptr_useful"]
    assert sum(b["csr_sectors"] for b in t["by_degree"]) == t["csr_sectors"]
    assert sum(b["edges"] for b in t["by_degree"]) == t["m_r"]
