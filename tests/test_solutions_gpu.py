"""Solutions 0-5 of SSSP_GPU()'s switch (apps/sssp/src/gpu/sssp_wrapper.cu:151-473:
thread queue, dual queue, shared / global delayed buffer, naive and per-block
nested launches) against the CPU oracle.

Every solution computes the same fixed point as the reference's unordered
frontier iteration, so distances must equal the restated heap Dijkstra of
SSSP_CPU (apps/sssp/src/cpu/sssp.cpp:13-47) bit for bit, whatever the race
order of the relaxations.  The cases follow the consolidation path's tests:
graph families, large-row thresholds, CTA shapes, the state form, the edge
cases of the CSR, malformed input and the host-side time bound.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOLUTIONS = [0, 1, 2, 3, 4, 5]


@pytest.fixture(scope="module")
def graphs(nps):
    return {
        "uniform": nps.gen_uniform(16384, 131072, 100, 1),
        "rmat16": nps.gen_rmat(16, 16, seed=3),
        "grid128": nps.gen_grid(128, 128, 0.05, 1000, 7),
    }


def _check(nps, oracle, g, sol, src=None, **kw):
    src = g.source if src is None else src
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, src)
    dist, st, info = nps.sssp_solution(g, sol, src, nps.Params(**kw))
    bad = np.nonzero(dist != ref)[0]
    assert bad.size == 0, f"solution {sol}: {bad.size} mismatches, first {bad[:5]} got {dist[bad[:5]]} want {ref[bad[:5]]}"
    assert st.status == 0
    assert st.reached == int((ref < nps.INF).sum())
    return st, info


@pytest.mark.parametrize("name", ["uniform", "rmat16", "grid128"])
@pytest.mark.parametrize("sol", SOLUTIONS)
def test_solution_matches_oracle(nps, oracle, cuda_device, graphs, sol, name):
    g = graphs[name]
    st, info = _check(nps, oracle, g, sol)
    assert st.iterations > 0 and st.vertices_processed >= st.reached
    if sol == 0:
        assert info.deferred == 0 and info.child_launches == 0
    assert info.host_reads >= 1


@pytest.mark.parametrize("thr", [1, 8, 64, 1 << 20])
@pytest.mark.parametrize("sol", SOLUTIONS)
def test_thresholds(nps, oracle, cuda_device, graphs, sol, thr):
    st, info = _check(nps, oracle, graphs["rmat16"], sol, threshold=thr)
    if sol > 0 and thr <= 64:
        assert info.deferred > 0  # R-MAT 16 has rows of 64+ edges on the frontier
    if thr == 1 << 20:
        assert info.deferred == 0 and info.child_launches == 0


@pytest.mark.parametrize("bs", [64, 192, 256, 1024])
@pytest.mark.parametrize("sol", SOLUTIONS)
def test_block_sizes(nps, oracle, cuda_device, graphs, sol, bs):
    _check(nps, oracle, graphs["uniform"], sol, block_size=bs, threshold=16)


@pytest.mark.parametrize("sol", [4, 5])
def test_nested_launches(nps, oracle, cuda_device, graphs, sol):
    """Large rows go to child grids; a launch the device runtime refuses is walked
    by its parent thread, so launches + fallbacks account for every deferral."""
    st, info = _check(nps, oracle, graphs["rmat16"], sol, threshold=32)
    assert info.deferred > 0
    assert info.child_launches + info.launch_fallbacks > 0
    if sol == 4:
        assert info.child_launches + info.launch_fallbacks == info.deferred
    else:
        assert info.child_launches + info.launch_fallbacks <= info.deferred


@pytest.mark.parametrize("sol", SOLUTIONS)
def test_edge_cases(nps, oracle, cuda_device, sol):
    g = nps.Graph(np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0, np.uint32))
    d, _, _ = nps.sssp_solution(g, sol, 0)
    assert d.tolist() == [0]
    g = nps.convertCSR(5, [1, 2], [2, 3], [4, 5])  # isolated source
    d, _, _ = nps.sssp_solution(g, sol, 0)
    assert d.tolist() == [0] + [nps.INF] * 4
    # 0 -> 1 (2^29), 1 -> 2 (2^29): the path length reaches 2^30 = INF
    g = nps.convertCSR(4, [0, 1, 0], [1, 2, 3], [1 << 29, 1 << 29, 0xFFFFFFFF])
    d, _, _ = nps.sssp_solution(g, sol, 0)
    assert d.tolist() == [0, 1 << 29, nps.INF, nps.INF]
    rng = np.random.default_rng(11)
    n, m = 3000, 40000
    s = rng.integers(0, n, m)
    t = np.where(rng.random(m) < 0.05, s, rng.integers(0, n, m))  # 5% self-loops
    w = rng.integers(0, 4, m)  # many zero weights
    _check(nps, oracle, nps.convertCSR(n, s, t, w), sol, int(s[0]), threshold=4)


@pytest.mark.parametrize("sol", SOLUTIONS)
def test_hub_star(nps, oracle, cuda_device, sol):
    # one row of 200k edges: walked by one thread (0), one CTA (1, 3), the whole
    # source CTA (2) or a child grid (4, 5)
    n = 200001
    s = np.zeros(n - 1, np.int32)
    t = np.arange(1, n, dtype=np.int32)
    w = (np.arange(n - 1) % 97 + 1).astype(np.uint32)
    _check(nps, oracle, nps.convertCSR(n, s, t, w), sol, 0)


def _dev(torch, a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)


@pytest.mark.parametrize("sol", SOLUTIONS + [6])
def test_state_form(nps, oracle, cuda_device, sol):
    """The state prepare_gpu() leaves (and arbitrary states): costs updated in
    place, every flag cleared."""
    import torch
    rng = np.random.default_rng(2 + sol)
    g = nps.gen_rmat(12, 8, seed=9)
    dev = cuda_device
    row, col, w = _dev(torch, g.row_ptr, dev), _dev(torch, g.col, dev), _dev(torch, g.w, dev)
    for trial in range(3):
        if trial == 0:
            cost = np.full(g.n, nps.INF, np.uint32)
            upd = np.zeros(g.n, np.uint8)
            cost[g.source], upd[g.source] = 0, 1
        else:
            cost = np.where(rng.random(g.n) < 0.3, rng.integers(0, 3000, g.n), nps.INF).astype(np.uint32)
            upd = (rng.random(g.n) < 0.05).astype(np.uint8)
        want_c, _ = oracle.sssp_state(g.row_ptr, g.col, g.w, cost, upd)
        d_cost, d_upd = _dev(torch, cost, dev), torch.from_numpy(upd).to(dev)
        st, _ = nps.sssp_solution_state(sol, row, col, w, d_cost, d_upd, g.n, g.m,
                                        nps.Params(threshold=[64, 8, 1][trial]))
        torch.cuda.synchronize()
        assert (d_cost.cpu().numpy().view(np.uint32) == want_c).all()
        assert int(d_upd.sum()) == 0


@pytest.mark.parametrize("sol", SOLUTIONS)
def test_SSSP_GPU_dispatch(nps, oracle, cuda_device, graphs, sol):
    g = graphs["uniform"]
    cost = nps.SSSP_GPU(g, solution=sol)
    assert cost.dtype == np.int32
    assert (cost.view(np.uint32) == oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)).all()


@pytest.mark.parametrize("sol", SOLUTIONS)
def test_malformed_csr_is_reported_not_faulted(nps, oracle, cuda_device, sol):
    import torch
    dev = cuda_device
    g = nps.gen_uniform(1000, 8000, 10, 3)
    w = _dev(torch, g.w, dev)
    bad_col = g.col.copy()
    bad_col[123] = 5000  # neighbour id beyond n
    for row_arr, col_arr in ((g.row_ptr, bad_col), (np.where(np.arange(g.n + 1) == 10, g.m + 100, g.row_ptr),
                                                    g.col)):
        cost = np.full(g.n, nps.INF, np.uint32)
        upd = np.ones(g.n, np.uint8)  # every row is walked
        cost[:] = 0
        with pytest.raises(nps.NpsError) as ei:
            nps.sssp_solution_state(sol, _dev(torch, row_arr.astype(np.int32), dev), _dev(torch, col_arr, dev), w,
                                    _dev(torch, cost, dev), torch.from_numpy(upd).to(dev), g.n, g.m,
                                    nps.Params(threshold=4))
        assert ei.value.status == 7  # NPS_ERR_FORMAT
    _check(nps, oracle, g, sol, 0)  # the context is still usable


def test_time_bound(nps, oracle, cuda_device, graphs):
    """timeout_s bounds the whole call on the host: a high-diameter grid needs far
    more iterations than fit in 1 us; the next call still works."""
    g = graphs["grid128"]
    with pytest.raises(nps.NpsError) as ei:
        nps.sssp_solution(g, 0, g.source, nps.Params(timeout_s=1e-6))
    assert ei.value.status == 4  # NPS_ERR_TIMEOUT
    _check(nps, oracle, g, 0)


def test_solution_6_is_consolidation(nps, oracle, cuda_device, graphs):
    g = graphs["rmat16"]
    d6, st, info = nps.sssp_solution(g, 6, g.source, nps.Params(level=2))
    d, _ = nps.sssp(g, g.source, nps.Params(level=2))
    assert (d6 == d).all() and info.deferred == 0
