"""GPU degree statistics (nps_degree_stats) against the reference analyzer's
goldens and the oracle restatement; host and device inputs, edge cases and
malformed offsets."""
import ctypes as C
import importlib
import json
import os

import numpy as np
import pytest

from test_degree_cpu import GOLD, graph_of, matches_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(GOLD))
def test_gpu_matches_the_reference_analyzer(nps, cuda_device, name):
    rec = GOLD[name]
    g = graph_of(nps, name, rec)
    matches_golden(nps.degree_stats(g), rec)


@pytest.mark.parametrize("kind", ["rmat18", "grid256", "star", "uniform"])
def test_gpu_matches_the_oracle(nps, oracle, cuda_device, kind):
    import torch
    if kind == "rmat18":
        g = nps.gen_rmat(18, 16, seed=4)
    elif kind == "grid256":
        g = nps.gen_grid(256, 256, 0.05, 1000, 2)
    elif kind == "star":  # one row of 5000 and 5000 empty rows: degree beyond the shared bins
        g = nps.convertCSR(5001, [0] * 5000, list(range(1, 5001)), [1] * 5000)
    else:
        g = nps.gen_uniform(1 << 16, 1 << 19, 100, 5)
    want = oracle.degree_stats(g.row_ptr)
    for arg in (g, torch.from_numpy(g.row_ptr.view(np.int32)).to(cuda_device)):
        got = nps.degree_stats(arg)
        for k in ("n", "m", "total_degree", "edges_by_degree", "max_degree", "min_degree", "max_degree_node",
                  "min_degree_node", "bins"):
            assert got[k] == want[k], k
        assert got["avg_degree"] == want["avg_degree"]
        assert np.array_equal(got["dist"], want["dist"])


def test_edge_cases_and_errors(nps, cuda_device):
    st = nps.degree_stats(np.array([0, 0], np.int32))  # one vertex, no edges
    assert (st["n"], st["m"], st["max_degree"], st["min_degree"], st["max_degree_node"]) == (1, 0, 0, 0, 0)
    assert list(st["dist"]) == [1]
    with pytest.raises(nps.NpsError) as ei:
        nps.degree_stats(np.array([0, 4, 2, 6], np.int32))  # decreasing offsets
    assert ei.value.status == 7
    info = nps.nps_degree_info()
    row = np.array([0, 3, 3, 5], np.int32)
    small = np.zeros(2, np.int64)  # max degree is 3: needs 4 slots
    rc = nps.lib.nps_degree_stats(row.ctypes.data, 3, 0, 0, C.byref(info), small.ctypes.data, 2)
    assert rc == 3 and info.max_degree == 3 and info.max_degree_node == 0
