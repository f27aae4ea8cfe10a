"""Parity of the persistent B200 SSSP kernel against the CPU oracle.

Every case compares distances bit-exactly with the restated heap Dijkstra of
SSSP_CPU (apps/sssp/src/cpu/sssp.cpp:13-47) on the same seeded inputs, across
consolidation levels (CONSOLIDATE_LEVEL 0/1/2 and hybrid), bucket widths
(delta = 0 is the reference's unordered frontier), block shapes and entry points.
"""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(nps, **kw):
    return nps.Params(**kw)


@pytest.fixture(scope="module")
def uniform(nps):
    return nps.gen_uniform(16384, 131072, 100, 1)


@pytest.fixture(scope="module")
def rmat16(nps):
    return nps.gen_rmat(16, 16, seed=3)


@pytest.fixture(scope="module")
def grid128(nps):
    return nps.gen_grid(128, 128, 0.05, 1000, 7)


def _check(nps, oracle, g, src, params):
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, src)
    dist, st = nps.sssp(g, src, params)
    bad = np.nonzero(dist != ref)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]} got {dist[bad[:5]]} want {ref[bad[:5]]}"
    return st


@pytest.mark.parametrize("level,delta", list(itertools.product([0, 1, 2, 3], [0, 1, 37, 100, 4096])))
def test_uniform_levels_deltas(nps, oracle, cuda_device, uniform, level, delta):
    st = _check(nps, oracle, uniform, 0, _p(nps, level=level, delta=delta))
    assert st.status == 0 and st.iterations > 0


@pytest.mark.parametrize("light_heavy", [False, True])
@pytest.mark.parametrize("level,delta", [(1, 7), (2, 32), (3, 255), (2, 1000)])
def test_light_heavy_split(nps, oracle, cuda_device, rmat16, grid128, light_heavy, level, delta):
    """Heavy edges (w >= delta) relaxed once per settled vertex must give the same distances."""
    for g in (rmat16, grid128):
        st = _check(nps, oracle, g, g.source, _p(nps, level=level, delta=delta, light_heavy=light_heavy,
                                                 threshold=32, block_threshold=128, grid_threshold=1024))
        assert st.status == 0


@pytest.mark.parametrize("bs", [128, 256, 512])
@pytest.mark.parametrize("level", [0, 1, 2])
def test_rmat_block_shapes(nps, oracle, cuda_device, rmat16, bs, level):
    _check(nps, oracle, rmat16, rmat16.source, _p(nps, level=level, block_size=bs, delta=64))


@pytest.mark.parametrize("thr", [1, 2, 8, 64, 1000])
def test_rmat_thresholds(nps, oracle, cuda_device, rmat16, thr):
    _check(nps, oracle, rmat16, rmat16.source,
           _p(nps, level=3, threshold=thr, block_threshold=max(thr, 32), grid_threshold=max(thr, 512), delta=16))


@pytest.mark.parametrize("delta", [0, 500, 3000])
def test_grid_high_diameter(nps, oracle, cuda_device, grid128, delta):
    st = _check(nps, oracle, grid128, 0, _p(nps, level=1, delta=delta))
    if delta:
        assert st.buckets > 0


def test_random_sources(nps, oracle, cuda_device, rmat16):
    rng = np.random.default_rng(5)
    for src in rng.integers(0, rmat16.n, 6):
        _check(nps, oracle, rmat16, int(src), _p(nps, level=2, delta=32))


def test_ctas_per_sm_and_repeat(nps, oracle, cuda_device, uniform):
    for cps in (1, 2):
        for _ in range(3):  # stamps carried across runs on one workspace
            _check(nps, oracle, uniform, 0, _p(nps, ctas_per_sm=cps, delta=10))


# ---- edge cases the reference's inputs can contain --------------------------

def test_single_vertex_and_empty(nps, cuda_device):
    g = nps.Graph(np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0, np.uint32))
    d, st = nps.sssp(g, 0)
    assert d.tolist() == [0]


def test_isolated_source(nps, oracle, cuda_device):
    g = nps.convertCSR(5, [1, 2], [2, 3], [4, 5])
    d, _ = nps.sssp(g, 0)
    assert d.tolist() == [0] + [nps.INF] * 4


def test_multi_edges_self_loops_zero_weights(nps, oracle, cuda_device):
    rng = np.random.default_rng(11)
    n, m = 3000, 40000
    s = rng.integers(0, n, m)
    t = np.where(rng.random(m) < 0.05, s, rng.integers(0, n, m))  # 5% self-loops
    w = rng.integers(0, 4, m)  # many zero weights
    g = nps.convertCSR(n, s, t, w)
    for lv, de in ((0, 0), (1, 1), (2, 2), (3, 7)):
        _check(nps, oracle, g, int(s[0]), _p(nps, level=lv, delta=de, threshold=4, block_threshold=16,
                                             grid_threshold=64))


def test_weights_near_inf_are_unreachable(nps, oracle, cuda_device):
    # 0 -> 1 (2^29), 1 -> 2 (2^29): the path length reaches 2^30 = INF
    g = nps.convertCSR(4, [0, 1, 0], [1, 2, 3], [1 << 29, 1 << 29, 0xFFFFFFFF])
    d, _ = nps.sssp(g, 0)
    assert d.tolist() == [0, 1 << 29, nps.INF, nps.INF]
    assert (d == oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)).all()


def test_hub_star_grid_tier(nps, oracle, cuda_device):
    # one vertex of degree 200k exercises the grid tier's chunk space
    n = 200001
    s = np.zeros(n - 1, np.int32)
    t = np.arange(1, n, dtype=np.int32)
    w = (np.arange(n - 1) % 97 + 1).astype(np.uint32)
    g = nps.convertCSR(n, s, t, w)
    for lv in (0, 1, 2):
        _check(nps, oracle, g, 0, _p(nps, level=lv))


# ---- device-pointer entry points ------------------------------------------------

def _dev(torch, a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)


def test_device_pointers_and_unaligned_columns(nps, oracle, cuda_device, rmat16):
    import torch
    g = rmat16
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    row = _dev(torch, g.row_ptr, cuda_device)
    # column / weight arrays starting 4 bytes past a 16-byte boundary: scalar path
    col = torch.zeros(g.m + 1, dtype=torch.int32, device=cuda_device)
    w = torch.zeros(g.m + 1, dtype=torch.int32, device=cuda_device)
    col[1:] = _dev(torch, g.col, cuda_device)
    w[1:] = _dev(torch, g.w, cuda_device)
    dist = torch.empty(g.n, dtype=torch.int32, device=cuda_device)
    for off in (0, 1):
        c = col[off:] if off else _dev(torch, g.col, cuda_device)
        ww = w[off:] if off else _dev(torch, g.w, cuda_device)
        st = nps.sssp_device(row, c, ww, g.n, g.m, g.source, dist, nps.Params(level=2, delta=50))
        torch.cuda.synchronize()
        assert (dist.cpu().numpy().view(np.uint32) == ref).all()
        assert st.status == 0


def test_consolidate_state_form(nps, oracle, cuda_device, uniform):
    """sssp_np_consolidate_gpu on the state prepare_gpu() leaves behind."""
    import torch
    g = uniform
    dev = cuda_device
    row, col, w = _dev(torch, g.row_ptr, dev), _dev(torch, g.col, dev), _dev(torch, g.w, dev)
    cost = np.full(g.n, nps.INF, np.uint32)
    upd = np.zeros(g.n, np.uint8)
    cost[0] = 0
    upd[0] = 1
    for level in (0, 1, 2):
        d_cost = _dev(torch, cost, dev)
        d_upd = torch.from_numpy(upd).to(dev)
        st = nps.sssp_np_consolidate_gpu(row, col, w, d_cost, d_upd, g.n, g.m, level=level)
        torch.cuda.synchronize()
        assert (d_cost.cpu().numpy().view(np.uint32) == oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)).all()
        assert int(d_upd.sum()) == 0 and st.iterations > 0


def test_state_form_arbitrary_state(nps, oracle, cuda_device):
    import torch
    rng = np.random.default_rng(2)
    g = nps.gen_rmat(12, 8, seed=9)
    dev = cuda_device
    row, col, w = _dev(torch, g.row_ptr, dev), _dev(torch, g.col, dev), _dev(torch, g.w, dev)
    for trial in range(4):
        cost = np.where(rng.random(g.n) < 0.3, rng.integers(0, 3000, g.n), nps.INF).astype(np.uint32)
        upd = (rng.random(g.n) < 0.05).astype(np.uint8)
        want_c, want_u = oracle.sssp_state(g.row_ptr, g.col, g.w, cost, upd)
        d_cost, d_upd = _dev(torch, cost, dev), torch.from_numpy(upd).to(dev)
        nps.sssp_np_consolidate_gpu(row, col, w, d_cost, d_upd, g.n, g.m,
                                    params=nps.Params(level=trial % 3, delta=[0, 64, 0, 200][trial]))
        torch.cuda.synchronize()
        assert (d_cost.cpu().numpy().view(np.uint32) == want_c).all()
        assert int(d_upd.sum()) == 0


def test_SSSP_GPU_mirror(nps, oracle, cuda_device, uniform):
    cost = nps.SSSP_GPU(uniform, level=nps.CONSOLIDATE_BLOCK)
    assert cost.dtype == np.int32
    assert (cost.view(np.uint32) == oracle.sssp_heap(uniform.row_ptr, uniform.col, uniform.w, 0)).all()
    with pytest.raises(nps.NpsError):
        nps.SSSP_GPU(uniform, solution=7)  # the reference's switch has cases 0-6
    assert (nps.SSSP_GPU(uniform, solution=3) == cost).all()


# ---- batch -------------------------------------------------------------------

def test_batch_uneven_instances(nps, oracle, cuda_device):
    import torch
    dev = cuda_device
    rng = np.random.default_rng(4)
    graphs, insts, keep = [], [], []
    for i in range(12):
        g = nps.gen_rmat(int(rng.integers(8, 14)), int(rng.choice([4, 8, 16, 32])), seed=100 + i)
        src = int(rng.integers(0, g.n))
        row, col, w = _dev(torch, g.row_ptr, dev), _dev(torch, g.col, dev), _dev(torch, g.w, dev)
        dist = torch.empty(g.n, dtype=torch.int32, device=dev)
        keep.append((row, col, w, dist))
        graphs.append((g, src))
        insts.append(nps.Instance(row, col, w, dist, g.n, g.m, src))
    for use_graph in (False, True, True):
        stats, ms = nps.sssp_batch(insts, nps.Params(level=3, delta=32, threshold=32, block_threshold=256,
                                                     grid_threshold=2048), use_graph=use_graph)
        torch.cuda.synchronize()
        for (g, src), (_, _, _, dist), st in zip(graphs, keep, stats):
            assert st.status == 0
            assert (dist.cpu().numpy().view(np.uint32) == oracle.sssp_heap(g.row_ptr, g.col, g.w, src)).all()
        assert ms > 0


# ---- failure detection (bounded waits, bad inputs) ---------------------------

def test_bounded_wait_times_out_and_context_survives(nps, oracle, cuda_device, uniform):
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp(uniform, 0, nps.Params(fault_inject_wait=True, timeout_s=0.2))
    assert ei.value.status == 4  # NPS_ERR_TIMEOUT
    _check(nps, oracle, uniform, 0, nps.Params())


def test_malformed_csr_is_reported_not_faulted(nps, oracle, cuda_device):
    import torch
    dev = cuda_device
    g = nps.gen_uniform(1000, 8000, 10, 3)
    bad_col = g.col.copy()
    bad_col[123] = 5000  # neighbour id beyond n
    row, col, w = _dev(torch, g.row_ptr, dev), _dev(torch, bad_col, dev), _dev(torch, g.w, dev)
    dist = torch.empty(g.n, dtype=torch.int32, device=dev)
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp_device(row, col, w, g.n, g.m, 0, dist)
    assert ei.value.status == 7  # NPS_ERR_FORMAT
    bad_row = g.row_ptr.copy()
    bad_row[10] = g.m + 100
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp_device(_dev(torch, bad_row, dev), _dev(torch, g.col, dev), w, g.n, g.m, 0, dist)
    assert ei.value.status == 7
    _check(nps, oracle, g, 0, nps.Params())


def test_invalid_arguments(nps, cuda_device, uniform):
    for kw in ({"level": 7}, {"block_size": 96}, {"threshold": 0}, {"timeout_s": 0.0}, {"order_degree": -1}):
        with pytest.raises(nps.NpsError) as ei:
            nps.sssp(uniform, 0, nps.Params(**kw))
        assert ei.value.status == 1
    with pytest.raises(nps.NpsError):
        nps.sssp(uniform, uniform.n)  # source out of range


@pytest.mark.parametrize("rounds", [1, 3, 16])
@pytest.mark.parametrize("level,delta,lh", [(2, 0, False), (3, 40, True), (1, 300, False), (0, 16, True)])
def test_warp_local_rounds(nps, oracle, cuda_device, rmat16, grid128, rounds, level, delta, lh):
    """Vertices a warp improves are processed by that warp within the same
    iteration for up to `rounds` rounds; distances must not change."""
    for g in (rmat16, grid128):
        _check(nps, oracle, g, g.source, _p(nps, level=level, delta=delta, light_heavy=lh, local_rounds=rounds,
                                           threshold=32, block_threshold=128, grid_threshold=1024))


@pytest.mark.parametrize("order_degree", [1, 4, 32, 100000])
@pytest.mark.parametrize("level,delta,lh", [(2, 16, False), (2, 64, True), (3, 5, True), (1, 300, False)])
def test_order_degree(nps, oracle, cuda_device, rmat16, grid128, order_degree, level, delta, lh):
    """Improved vertices below order_degree join the current bucket whatever their
    distance (only larger rows wait for their bucket); distances must not change."""
    for g in (rmat16, grid128):
        _check(nps, oracle, g, g.source, _p(nps, level=level, delta=delta, light_heavy=lh, order_degree=order_degree,
                                           threshold=32, block_threshold=128, grid_threshold=1024))


def test_grid_tier_small_threshold_items(nps, oracle, cuda_device, rmat16, uniform):
    """Grid tier with threshold 1: rows of one chunk, so a work item spans many
    list entries (several 32-entry windows per item)."""
    for g in (rmat16, uniform):
        for delta in (0, 50):
            _check(nps, oracle, g, g.source, _p(nps, level=2, threshold=1, delta=delta))


@pytest.mark.parametrize("first,rest", [([2], 10), ([1, 1], 6), ([0, 3, 5, 2, 7, 1, 9], 4), ([], 1)])
@pytest.mark.parametrize("lh", [False, True])
def test_delta_schedule(nps, oracle, cuda_device, rmat16, grid128, first, rest, lh):
    """Per-bucket widths from Params.delta_schedule (the form a learned policy's
    decisions take): every schedule gives the oracle's distances."""
    word = nps.delta_schedule(first, rest)
    for g in (rmat16, grid128):
        st = _check(nps, oracle, g, g.source, _p(nps, level=2, delta_schedule=word, light_heavy=lh, threshold=32))
        assert st.buckets > 0


def test_delta_schedule_word():
    import importlib
    nps = importlib.import_module("nested-parallelism_b200")
    assert nps.delta_schedule([2], 10) == 0xAAAAAAA2
    assert nps.delta_schedule([], 3) == 0x33333333
    with pytest.raises(ValueError):
        nps.delta_schedule([16], 1)
