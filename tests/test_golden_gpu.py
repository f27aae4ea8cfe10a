"""The B200 kernel against the golden fixtures made by the reference's SSSP_CPU.

Bit-exact distance fingerprints for every golden case and every hand-made edge
case, under the consolidation levels and bucket widths of the API.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))
DISTS = np.load(os.path.join(HERE, "golden", "golden_dist.npz"))

PARAMS = [dict(level=0), dict(level=1), dict(level=2, delta=0), dict(level=2, delta=64),
          dict(level=3, delta=16, threshold=8, block_threshold=64, grid_threshold=512),
          dict(level=2, delta=300, light_heavy=False)]


def _gen(nps, case):
    a = case["args"]
    if case["kind"] == "uniform":
        return nps.gen_uniform(a["n"], a["m"], a["wmax"], a["seed"])
    if case["kind"] == "rmat":
        return nps.gen_rmat(a["scale"], a["edge_factor"], seed=a["seed"])
    return nps.gen_grid(a["rows"], a["cols"], a["drop"], a["wmax"], a["seed"])


@pytest.mark.parametrize("name", sorted(GOLD["cases"]))
def test_kernel_matches_reference_goldens(nps, cuda_device, name):
    case = GOLD["cases"][name]
    g = _gen(nps, case)
    for kw in PARAMS:
        d, st = nps.sssp(g, case["source"], nps.Params(**kw))
        assert nps.fnv1a(d) == case["dist_fnv1a"], (name, kw)
        if name in DISTS.files:
            assert np.array_equal(d, DISTS[name])
        assert st.status == 0


@pytest.mark.parametrize("name", sorted(GOLD["edge_cases"]))
def test_kernel_edge_cases(nps, cuda_device, name):
    c = GOLD["edge_cases"][name]
    g = nps.convertCSR(c["n"], c["src"], c["dst"], c["w"])
    for kw in PARAMS:
        d, _ = nps.sssp(g, c["source"], nps.Params(**kw))
        assert d.tolist() == c["dist"], (name, kw)


@pytest.mark.parametrize("fname", sorted(GOLD["readers"]))
def test_kernel_on_files_read_like_the_reference(nps, oracle, cuda_device, fname):
    readers = {0: nps.readInputDIMACS9, 1: nps.readInputDIMACS10, 2: nps.readInputSLNDC}
    g = readers[GOLD["readers"][fname]["format"]](os.path.join(HERE, "golden", fname))
    cost = nps.SSSP_GPU(g)
    assert np.array_equal(cost.view(np.uint32), oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source))
