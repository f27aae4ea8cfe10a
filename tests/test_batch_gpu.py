"""The batched workload on the GPU: 64 R-MAT instances (scale 12..18, edge
factor 4/8/16/32, w in [1,255], random sources) in one persistent launch
replayed from a CUDA graph, with parameters picked by the autotuner; every
instance bit-exact against the CPU Dijkstra oracle."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch64():
    B = importlib.import_module("nested-parallelism_b200.batch")
    return B.rmat_batch(64, seed=7)


@pytest.fixture(scope="module")
def want(batch64, oracle):
    return [oracle.sssp_heap(it.graph.row_ptr, it.graph.col, it.graph.w, it.source) for it in batch64]


def test_batch64_autotuned_graph_launch_is_exact(nps, oracle, cuda_device, batch64, want):
    import torch
    at = importlib.import_module("nested-parallelism_b200.autotune")
    dgs = [at.to_device(it.graph, it.source, cuda_device) for it in batch64]
    axes = {"level": [1, 2, 3], "threshold": [32, 64, 128], "delta": [0, 32, 128, 1024],
            "block_size": [256, 512]}
    best, ms, log = at.autotune(dgs, repeats=2, budget=16, axes=axes, batch=True)
    assert len(log) >= 2 and ms > 0
    insts = [nps.Instance(d.row_ptr, d.col, d.w, d.dist, d.n, d.m, d.src) for d in dgs]
    for use_graph in (True, True, False):
        for d in dgs:
            d.dist.fill_(-1)
        stats, kms = nps.sssp_batch(insts, best, use_graph=use_graph)
        torch.cuda.synchronize()
        assert kms > 0
        for d, st, ref in zip(dgs, stats, want):
            assert st.status == 0
            got = d.dist.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, ref)


def test_device_batch_results_match_the_oracle(nps, cuda_device, batch64, want):
    B = importlib.import_module("nested-parallelism_b200.batch")
    db = B.DeviceBatch(batch64[:20], cuda_device)
    stats, _ = db.run(nps.Params(level=2, delta=0, block_size=512))
    res = db.results()
    assert [r["index"] for r in res] == list(range(20))
    for r, ref, st in zip(res, want[:20], stats):
        assert r["fnv1a"] == nps.fnv1a(ref)
        assert r["reached"] == int((ref < nps.INF).sum()) == st.reached


def test_rebalanced_batch_stays_exact(nps, cuda_device, batch64, want):
    """Calls 2 and 3 on an unchanged instance set re-balance the teams' CTAs from the
    measured per-instance solve times (and re-capture the graph); every call, before
    and after, gives the oracle's distances, and each instance reports its solve time."""
    B = importlib.import_module("nested-parallelism_b200.batch")
    db = B.DeviceBatch(batch64, cuda_device)
    p = nps.Params(level=2, threshold=64, delta=0, block_size=512)
    for call in range(5):
        for k in db.keep:
            k[3].fill_(-1)
        stats, ms = db.run(p, use_graph=True)
        assert ms > 0
        assert all(st.status == 0 and st.kernel_ms > 0 for st in stats)
        for got, ref in zip(db.distances(), want):
            assert np.array_equal(got, ref), f"call {call}"
