"""Grid-tier rows sorted when their near-queue pushes are flushed
(nps_params.sort_at_push = 1), when they are taken from the queue (-1), or by the
grid threshold (0, the default): the distances must be those of SSSP_CPU
(apps/sssp/src/cpu/sssp.cpp:13-47) in every case, on every graph family, level,
bucket width and block shape, in batches and under the learned policy.  With
sorting at push a vertex may reach the grid-tier list both as a pushed row and
as a queue or far-pile entry in the same iteration; the near stamp lets only one
of them in, which the power-law graphs exercise (many of their pushes are
grid-tier rows, and bucket widths above 0 send rows through the far pile).  The
hub graph adds one 120,000-edge row walked by the whole team.
"""
import importlib
import itertools
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "nested-parallelism_b200", "policy_weights.npz")


@pytest.fixture(scope="module")
def graphs(nps):
    n = 200_000
    rng = np.random.default_rng(12)
    src = np.concatenate([np.zeros(120_000, np.int64), rng.integers(0, n, 400_000)])
    dst = np.concatenate([rng.integers(1, n, 120_000), rng.integers(0, n, 400_000)])
    hub = nps.convertCSR(n, src, dst, rng.integers(1, 300, src.size))
    return {"uniform": nps.gen_uniform(16384, 131072, 100, 1), "rmat16": nps.gen_rmat(16, 16, seed=3),
            "grid128": nps.gen_grid(128, 128, 0.05, 1000, 7), "rmat18": nps.gen_rmat(18, 8, seed=11), "hub": hub}


def _check(nps, oracle, g, src, params):
    want = oracle.sssp_heap(g.row_ptr, g.col, g.w, src)
    dist, st = nps.sssp(g, src, params)
    bad = np.nonzero(dist != want)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]} got {dist[bad[:5]]} want {want[bad[:5]]}"
    assert st.status == 0
    return st


@pytest.mark.parametrize("name,sort", list(itertools.product(["uniform", "rmat16", "grid128", "rmat18", "hub"],
                                                             [1, -1, 0])))
@pytest.mark.parametrize("level,delta", [(2, 0), (2, 37), (3, 0), (3, 300), (1, 0)])
def test_sort_at_push_families_levels_widths(nps, oracle, cuda_device, graphs, name, sort, level, delta):
    g = graphs[name]
    src = 0 if name == "hub" else g.source
    _check(nps, oracle, g, src, nps.Params(level=level, delta=delta, threshold=16, block_threshold=64,
                                           grid_threshold=256, block_size=512, light_heavy=False,
                                           sort_at_push=sort))


@pytest.mark.parametrize("bs,thr", [(128, 4), (256, 32), (512, 1)])
def test_sort_at_push_block_shapes_and_thresholds(nps, oracle, cuda_device, graphs, bs, thr):
    for name in ("rmat16", "hub"):
        g = graphs[name]
        src = 0 if name == "hub" else g.source
        _check(nps, oracle, g, src, nps.Params(level=2, delta=0, threshold=thr, block_size=bs, sort_at_push=1))


def test_sort_at_push_fewer_iterations_same_distances(nps, oracle, cuda_device, graphs):
    """On the power-law graph at the grid level, sorting at push walks a grid-tier row
    one iteration after it is found instead of two."""
    g = graphs["rmat18"]
    p = dict(level=2, delta=0, threshold=16, block_size=512)
    on = _check(nps, oracle, g, g.source, nps.Params(sort_at_push=1, **p))
    off = _check(nps, oracle, g, g.source, nps.Params(sort_at_push=-1, **p))
    assert on.iterations < off.iterations


def test_sort_at_push_in_a_batch(nps, oracle, cuda_device):
    import torch
    B = importlib.import_module("nested-parallelism_b200.batch")
    at = importlib.import_module("nested-parallelism_b200.autotune")
    items = B.rmat_batch(12, seed=21)
    dgs = [at.to_device(it.graph, it.source, cuda_device) for it in items]
    insts = [nps.Instance(d.row_ptr, d.col, d.w, d.dist, d.n, d.m, d.src) for d in dgs]
    for sort in (1, -1, 0):
        for d in dgs:
            d.dist.fill_(-1)
        stats, _ = nps.sssp_batch(insts, nps.Params(level=2, threshold=16, delta=0, block_size=512,
                                                    sort_at_push=sort), use_graph=False)
        torch.cuda.synchronize()
        for it, d, st in zip(items, dgs, stats):
            assert st.status == 0
            want = oracle.sssp_heap(it.graph.row_ptr, it.graph.col, it.graph.w, it.source)
            assert np.array_equal(d.dist.cpu().numpy().view(np.uint32), want)


def test_sort_at_push_under_the_learned_policy(nps, oracle, cuda_device, graphs):
    pol = importlib.import_module("nested-parallelism_b200.policy")
    pol.load_into_kernel(pol.MLPWeights.load(WEIGHTS), 0)
    for name in ("rmat16", "rmat18", "grid128", "hub"):
        g = graphs[name]
        src = 0 if name == "hub" else g.source
        for sort in (1, -1):
            _check(nps, oracle, g, src, nps.Params(level=2, threshold=32, block_size=512, light_heavy=False,
                                                   policy=nps.POLICY_LEARNED, policy_min_edges=-1, trace=True,
                                                   sort_at_push=sort))


def test_sort_at_push_rejects_other_values(nps, cuda_device, graphs):
    with pytest.raises(nps.NpsError):
        nps.sssp(graphs["uniform"], 0, nps.Params(sort_at_push=2))
