"""The asynchronous bucket schedule (nps_params.schedule = NPS_SCHEDULE_ASYNC)
against the CPU oracle's Dijkstra, bit for bit.

Inside a bucket the persistent kernel has no barrier: improved vertices and
256-edge row segments go to device work rings that every warp drains as work
appears, and the team meets only when a bucket's pending total reaches zero.
The distances must be those of SSSP_CPU (apps/sssp/src/cpu/sssp.cpp:13-47) on
every graph family, bucket width, threshold and block shape, on repeated runs
over the same persistent rings, in the state form and after a run that stopped
on a timeout.
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
    return {"uniform": nps.gen_uniform(16384, 131072, 100, 1), "rmat16": nps.gen_rmat(16, 16, seed=3),
            "grid128": nps.gen_grid(128, 128, 0.05, 1000, 7), "rmat18": nps.gen_rmat(18, 8, seed=11)}


def _async(nps, **kw):
    kw.setdefault("level", nps.CONSOLIDATE_GRID)
    kw.setdefault("light_heavy", False)
    kw.setdefault("timeout_s", 5.0)
    return nps.Params(schedule=nps.SCHEDULE_ASYNC, **kw)


def _check(nps, oracle, g, src, params):
    want = oracle.sssp_heap(g.row_ptr, g.col, g.w, src)
    dist, st = nps.sssp(g, src, params)
    bad = np.nonzero(dist != want)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]} got {dist[bad[:5]]} want {want[bad[:5]]}"
    assert st.status == 0
    return st


@pytest.mark.parametrize("name,delta", list(itertools.product(["uniform", "rmat16", "grid128", "rmat18"],
                                                              [0, 1, 37, 4096])))
def test_async_families_and_widths(nps, oracle, cuda_device, graphs, name, delta):
    g = graphs[name]
    st = _check(nps, oracle, g, g.source, _async(nps, delta=delta, threshold=32, block_size=512))
    if delta == 0:
        assert st.iterations == 1  # one bucket: no barrier between frontiers


@pytest.mark.parametrize("thr,bs", [(1, 256), (4, 512), (64, 128), (1 << 20, 512)])
def test_async_thresholds_and_block_shapes(nps, oracle, cuda_device, graphs, thr, bs):
    for name in ("rmat16", "uniform"):
        g = graphs[name]
        _check(nps, oracle, g, g.source, _async(nps, delta=16, threshold=thr, block_size=bs))


def test_async_repeated_runs_on_persistent_rings(nps, oracle, cuda_device, graphs):
    """Ring heads, tails and slot tags carry over from run to run (and wrap around
    the ring many times); every run stays exact."""
    g = graphs["rmat16"]
    rng = np.random.default_rng(3)
    for i, src in enumerate(rng.integers(0, g.n, 12)):
        _check(nps, oracle, g, int(src), _async(nps, delta=[0, 8, 300][i % 3], threshold=[8, 32][i % 2]))


def test_async_hub_segments(nps, oracle, cuda_device):
    """A 300,000-edge hub is cut into 1,172 segments that every warp shares."""
    n = 400_000
    rng = np.random.default_rng(9)
    src = np.concatenate([np.zeros(300_000, np.int64), rng.integers(0, n, 600_000)])
    dst = np.concatenate([rng.integers(1, n, 300_000), rng.integers(0, n, 600_000)])
    w = rng.integers(1, 200, src.size)
    g = nps.convertCSR(n, src, dst, w)
    for _ in range(4):  # repeated: the interleaving of pushes and takes differs from run to run
        _check(nps, oracle, g, 0, _async(nps, delta=0, threshold=64))
        _check(nps, oracle, g, 0, _async(nps, delta=50, threshold=256))


def test_async_learned_policy(nps, oracle, cuda_device, graphs):
    pol = importlib.import_module("nested-parallelism_b200.policy")
    pol.load_into_kernel(pol.MLPWeights.load(WEIGHTS), 0)
    for name in ("rmat16", "rmat18", "grid128"):
        g = graphs[name]
        _check(nps, oracle, g, g.source, _async(nps, policy=nps.POLICY_LEARNED, threshold=32, block_size=512, policy_min_edges=-1))


def test_async_state_form(nps, oracle, cuda_device, graphs):
    import torch
    g = graphs["rmat16"]
    rng = np.random.default_rng(4)
    cost = np.full(g.n, oracle.INF, np.uint32)
    upd = np.zeros(g.n, np.uint8)
    seeds = rng.integers(0, g.n, 50)
    cost[seeds] = rng.integers(0, 500, 50).astype(np.uint32)
    upd[seeds] = 1
    want, _ = oracle.sssp_state(g.row_ptr, g.col, g.w, cost, upd)
    dev = cuda_device
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)
    d_cost = t(cost)
    d_upd = torch.from_numpy(upd.copy()).to(dev)
    st = nps.sssp_np_consolidate_gpu(t(g.row_ptr), t(g.col), t(g.w), d_cost, d_upd, g.n, g.m,
                                     params=_async(nps, delta=32, threshold=16))
    assert st.status == 0
    assert np.array_equal(d_cost.cpu().numpy().view(np.uint32), want)
    assert not d_upd.cpu().numpy().any()


def test_async_exact_after_a_run_that_timed_out(nps, oracle, cuda_device, graphs):
    g = graphs["uniform"]
    with pytest.raises(nps.NpsError):
        nps.sssp(g, 0, _async(nps, delta=16, timeout_s=0.5, fault_inject_wait=True))
    _check(nps, oracle, g, 0, _async(nps, delta=16))


def test_async_falls_back_to_iterations_when_not_eligible(nps, oracle, cuda_device, graphs):
    """Block level, or a light/heavy split in effect, run the iteration schedule."""
    g = graphs["rmat16"]
    st = _check(nps, oracle, g, g.source, _async(nps, level=nps.CONSOLIDATE_BLOCK, delta=0))
    assert st.iterations > 1
    st = _check(nps, oracle, g, g.source, _async(nps, delta=64, light_heavy=True))
    assert st.iterations > 1
