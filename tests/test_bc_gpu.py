"""Betweenness centrality on the GPU (nps_bc, the bc application's
bc_np_consolidate_gpu) against the reference's bc_cpu: the golden centralities it
produced, and the oracle's restatement on larger graphs and source subsets.  The
GPU rounds every step as the reference does and folds sources in order, so every
comparison is bit for bit -- except the payload of a NaN (path counts that wrap
can give 0/0): x86 writes 0xFFC00000 where the GPU writes 0x7FFFFFFF, so NaNs
compare as NaNs."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

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


def _same(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    bits = a.view(np.uint32) == b.view(np.uint32)
    return bool(np.all(bits | (np.isnan(a) & np.isnan(b))))


def test_golden_centralities(nps, cuda_device, golden, oracle):
    for name, case in golden["bc"]["cases"].items():
        g = _gen(nps, case["kind"], case["args"])
        b, st = nps.bc(g)
        assert oracle.fnv1a(b.view(np.uint32)) == case["bc_fnv1a"], name
        assert st.status == 0 and st.vertices_processed == g.n


def test_golden_edge_cases(nps, cuda_device, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        b, _ = nps.bc(g)
        assert b.tolist() == golden["bc"]["edge_cases"][name], name


@pytest.mark.parametrize("kind", ["rmat14", "grid96", "uniform8k", "star"])
def test_larger_graphs_source_subsets(nps, oracle, cuda_device, kind):
    rng = np.random.default_rng(3)
    if kind == "rmat14":
        g = nps.gen_rmat(14, 16, seed=5)
    elif kind == "grid96":
        g = nps.gen_grid(96, 96, 0.05, 10, 2)
    elif kind == "uniform8k":
        g = nps.gen_uniform(8192, 65536, 10, 4)
    else:  # a 20k-edge hub: its forward row is walked by a warp, its backward row by one thread
        n = 20001
        s = np.concatenate([np.zeros(n - 1, np.int64), np.arange(1, n)])
        t = np.concatenate([np.arange(1, n), (np.arange(1, n) * 7) % n])
        g = nps.convertCSR(n, s, t, np.ones(s.shape[0], np.uint32))
    for sources in (np.arange(min(g.n, 600)), rng.integers(0, g.n, 300), np.array([g.n - 1, 0, g.n - 1])):
        b, _ = nps.bc(g, sources)
        assert _same(b, oracle.bc(g.row_ptr, g.col, sources)), (kind, sources[:5])


def test_many_blocks_of_sources(nps, oracle, cuda_device):
    """More sources than one block of dependency rows holds (blocks fold in order)."""
    g = nps.gen_rmat(12, 8, seed=9)
    want = oracle.bc(g.row_ptr, g.col)
    for per_block in (7, 296, 1000):
        b, _ = nps.bc(g, params=nps.Params(bc_block_sources=per_block))
        assert _same(b, want), per_block


def test_device_pointers(nps, oracle, cuda_device):
    import torch
    g = nps.gen_rmat(11, 8, seed=4)
    dev = cuda_device
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    src = torch.arange(0, g.n, 3, dtype=torch.int32, device=dev)
    st = nps.bc_device(row, col, g.n, g.m, out, src, int(src.numel()))
    torch.cuda.synchronize()
    assert _same(out.cpu().numpy(), oracle.bc(g.row_ptr, g.col, np.arange(0, g.n, 3))) and st.status == 0
    bad = torch.tensor([0, g.n], dtype=torch.int32, device=dev)
    with pytest.raises(nps.NpsError) as ei:
        nps.bc_device(row, col, g.n, g.m, out, bad, 2)
    assert ei.value.status == 1


def test_malformed_csr_is_reported_not_faulted(nps, oracle, cuda_device):
    import torch
    g = nps.gen_uniform(1000, 8000, 10, 3)
    dev = cuda_device
    bad = g.col.copy()
    bad[77] = 5000
    out = torch.empty(g.n, dtype=torch.float32, device=dev)
    with pytest.raises(nps.NpsError) as ei:
        nps.bc_device(torch.from_numpy(g.row_ptr.view(np.int32)).to(dev), torch.from_numpy(bad.view(np.int32)).to(dev),
                      g.n, g.m, out)
    assert ei.value.status == 7
    b, _ = nps.bc(g, np.arange(50))
    assert _same(b, oracle.bc(g.row_ptr, g.col, np.arange(50)))
