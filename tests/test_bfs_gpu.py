"""Breadth-first levels on the persistent SSSP engine (nps_bfs, the bfs-rec
application's bfs_rec_dp_cons_gpu) against the reference's bfs_cpu: the golden
levels it produced, and the oracle's restatement on larger graphs.  Levels are
integers, so every case is exact."""
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


CONFIGS = [dict(), dict(delta=0, level=1), dict(delta=0, level=0), dict(delta=2, level=3),
           dict(delta=1, level=2, block_size=512, threshold=16), dict(delta=1, level=1, local_rounds=3)]


@pytest.mark.parametrize("cfg", range(len(CONFIGS)))
def test_golden_levels(nps, cuda_device, golden, cfg):
    for name, case in golden["cases"].items():
        g = _gen(nps, case["kind"], case["args"])
        want = golden["bfs"]["cases"][name]
        lv, st = nps.bfs(g, want["source"], nps.bfs_params(**CONFIGS[cfg]))
        assert nps.fnv1a(lv.view(np.uint32)) == want["levels_fnv1a"], (name, CONFIGS[cfg])
        assert st.status == 0 and st.reached == want["n_reached"]


def test_golden_edge_cases(nps, cuda_device, golden):
    for name, case in golden["edge_cases"].items():
        g = nps.convertCSR(case["n"], case["src"], case["dst"], case["w"])
        for cfg in CONFIGS[:3]:
            lv, _ = nps.bfs(g, case["source"], nps.bfs_params(**cfg))
            assert lv.tolist() == golden["bfs"]["edge_cases"][name], (name, cfg)


@pytest.mark.parametrize("kind", ["rmat18", "grid512", "star"])
def test_larger_graphs_against_the_oracle(nps, oracle, cuda_device, kind):
    if kind == "rmat18":
        g = nps.gen_rmat(18, 16, seed=11)
    elif kind == "grid512":
        g = nps.gen_grid(512, 512, 0.05, 1000, 2)
    else:  # one row of 300k edges: the grid tier's chunk space
        n = 300001
        g = nps.convertCSR(n, np.zeros(n - 1, np.int32), np.arange(1, n, dtype=np.int32), np.ones(n - 1, np.uint32))
    want = oracle.bfs_levels(g.row_ptr, g.col, g.source)
    for cfg in (dict(), dict(delta=0, level=2), dict(delta=1, level=1)):
        lv, st = nps.bfs(g, g.source, nps.bfs_params(**cfg))
        bad = np.nonzero(lv != want)[0]
        assert bad.size == 0, (cfg, bad[:5], lv[bad[:5]], want[bad[:5]])


def test_device_pointers_and_unaligned_columns(nps, oracle, cuda_device):
    import torch
    g = nps.gen_rmat(16, 16, seed=3)
    want = oracle.bfs_levels(g.row_ptr, g.col, g.source)
    dev = cuda_device
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.zeros(g.m + 1, dtype=torch.int32, device=dev)
    col[1:] = torch.from_numpy(g.col.view(np.int32)).to(dev)
    level = torch.empty(g.n, dtype=torch.int32, device=dev)
    for c in (torch.from_numpy(g.col.view(np.int32)).to(dev), col[1:]):
        st = nps.bfs_device(row, c, g.n, g.m, g.source, level)
        torch.cuda.synchronize()
        assert (level.cpu().numpy() == want).all() and st.status == 0


def test_bfs_does_not_disturb_weighted_runs(nps, oracle, cuda_device):
    """The engine's unit-weight mode is per call: a weighted SSSP right after a BFS
    on the same context reads its weights."""
    g = nps.gen_uniform(16384, 131072, 100, 1)
    lv, _ = nps.bfs(g, 0)
    d, _ = nps.sssp(g, 0, nps.Params(level=2, delta=64))
    assert (lv == oracle.bfs_levels(g.row_ptr, g.col, 0)).all()
    assert (d == oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)).all()
