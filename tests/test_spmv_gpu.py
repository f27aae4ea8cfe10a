"""y = A x on the GPU (nps_spmv, the SpMV application's spmv_np_consolidate_gpu)
against the reference.  With the reference's own data (val[i] = i % 13 + 0.5,
x[i] = i % 17 + 0.5) every sum is exact in double, so y must equal the
reference's spmv_omp bit for bit at every consolidation level.  With general
data the summation order differs from the reference's, so y is compared within
a relative 1e-12, and two runs of the same call must agree bit for bit (the
order is fixed by the matrix)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LEVELS = [0, 1, 2]


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


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("threshold", [1, 16, 64, 1 << 20])
def test_golden_y(nps, oracle, cuda_device, golden, level, threshold):
    for name, case in golden["cases"].items():
        g = _gen(nps, case["kind"], case["args"])
        val, x = oracle.spmv_data(g.n, g.m)
        y, st = nps.spmv(g, val, x, nps.Params(level=level, threshold=threshold))
        assert oracle.fnv1a(y.view(np.uint32)) == golden["spmv"]["cases"][name]["y_fnv1a"], (name, level)
        assert st.status == 0


def test_golden_edge_cases(nps, oracle, cuda_device, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        val, x = oracle.spmv_data(g.n, g.m)
        for level in LEVELS:
            y, _ = nps.spmv(g, val, x, nps.Params(level=level, threshold=2))
            assert y.tolist() == golden["spmv"]["edge_cases"][name], (name, level)


@pytest.mark.parametrize("level", LEVELS)
def test_long_rows_and_empty_rows(nps, oracle, cuda_device, level):
    """A 300k-nonzero row (147 grid-level chunks), rows of every length up to
    5000, and empty rows between them."""
    rng = np.random.default_rng(4)
    n = 400000
    lens = np.zeros(n, np.int64)
    lens[7] = 300000
    lens[1000:6000] = rng.integers(0, 5000, 5000)
    lens[10000:200000:3] = rng.integers(1, 40, len(range(10000, 200000, 3)))
    src = np.repeat(np.arange(n), lens)
    dst = rng.integers(0, n, src.shape[0])
    g = nps.convertCSR(n, src, dst, np.ones(src.shape[0], np.uint32))
    val, x = oracle.spmv_data(g.n, g.m)
    y, _ = nps.spmv(g, val, x, nps.Params(level=level))
    assert np.array_equal(y, oracle.spmv(g.row_ptr, g.col, val, x))


@pytest.mark.parametrize("level", LEVELS)
def test_general_data_is_close_and_repeatable(nps, oracle, cuda_device, level):
    g = nps.gen_rmat(17, 16, seed=5)
    rng = np.random.default_rng(level)
    val = rng.standard_normal(g.m)
    x = rng.standard_normal(g.n)
    y1, _ = nps.spmv(g, val, x, nps.Params(level=level, threshold=32))
    y2, _ = nps.spmv(g, val, x, nps.Params(level=level, threshold=32))
    assert np.array_equal(y1, y2)
    want = oracle.spmv(g.row_ptr, g.col, val, x)
    absrow = oracle.spmv(g.row_ptr, g.col, np.abs(val), np.abs(x))
    assert np.all(np.abs(y1 - want) <= 1e-12 * np.maximum(absrow, 1e-300))


def test_device_pointers(nps, oracle, cuda_device):
    import torch
    g = nps.gen_rmat(16, 16, seed=3)
    val, x = oracle.spmv_data(g.n, g.m)
    dev = cuda_device
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    dv, dx = torch.from_numpy(val).to(dev), torch.from_numpy(x).to(dev)
    dy = torch.empty(g.n, dtype=torch.float64, device=dev)
    for level in LEVELS:
        st = nps.spmv_device(row, col, dv, dx, dy, g.n, g.m, nps.Params(level=level))
        torch.cuda.synchronize()
        assert np.array_equal(dy.cpu().numpy(), oracle.spmv(g.row_ptr, g.col, val, x)) and st.status == 0


def test_malformed_csr_is_reported_not_faulted(nps, oracle, cuda_device):
    import torch
    g = nps.gen_uniform(1000, 8000, 10, 3)
    val, x = oracle.spmv_data(g.n, g.m)
    dev = cuda_device
    bad = g.col.copy()
    bad[77] = 5000
    dy = torch.empty(g.n, dtype=torch.float64, device=dev)
    for level in LEVELS:
        with pytest.raises(nps.NpsError) as ei:
            nps.spmv_device(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev),
                            torch.from_numpy(bad.view(np.int32)).to(dev), torch.from_numpy(val).to(dev),
                            torch.from_numpy(x).to(dev), dy, g.n, g.m, nps.Params(level=level, threshold=4))
        assert ei.value.status == 7
    y, _ = nps.spmv(g, val, x)
    assert np.array_equal(y, oracle.spmv(g.row_ptr, g.col, val, x))
