"""nps_sssp_noalloc, the entry point that allocates nothing.

Some callers of this library cannot allocate device memory at the moment they
ask for shortest paths: a service that has reserved all device memory in its own
pool, a host that forbids allocator calls from its callbacks.  nps_sssp_noalloc
serves them from a static device array sized for graphs of up to
NPS_NOALLOC_MAX_VERTICES vertices.  Its distances must equal the CPU oracle's
Dijkstra and the regular entry point's bit for bit (integer distances: zero
tolerance), and must stay equal on a second call in a row, since calls reuse
the same array.  The call synchronises its stream to return a status; on a
stream that is being captured it returns NPS_ERR_INVALID_ARG.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_VERTICES = 131072  # NPS_NOALLOC_MAX_VERTICES in include/nps.h
NPS_ERR_INVALID_ARG, NPS_ERR_CAPACITY, NPS_ERR_TIMEOUT = 1, 3, 4


def _dev(torch, a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)


def _noalloc(nps, row, col, w, n, m, src, out, params, stream=None):
    from importlib import import_module
    native = import_module("nested-parallelism_b200._native")
    p = params.to_c(device_ptrs=True, stream=stream)
    st = native.nps_stats()
    rc = nps.lib.nps_sssp_noalloc(row.data_ptr(), col.data_ptr(), w.data_ptr(), n, m, src, out.data_ptr(),
                                  C.byref(p), C.byref(st))
    return rc, st


def _solve(nps, torch, dev, row, col, w, g, src, params):
    out = torch.full((g.n,), -1, dtype=torch.int32, device=dev)
    rc, st = _noalloc(nps, row, col, w, g.n, g.m, src, out, params)
    assert rc == 0, nps.lib.nps_last_error_string().decode()
    assert st.status == 0 and st.iterations > 0
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32).copy()


@pytest.mark.parametrize("level,delta", [(2, 32), (1, 0), (3, 64)])
def test_noalloc_matches_oracle_and_nps_sssp_on_two_calls(nps, oracle, cuda_device, level, delta):
    import torch
    g = nps.gen_rmat(16, 16, seed=21)  # 65,536 vertices, inside the limit
    assert g.n <= NOALLOC_MAX_VERTICES
    row, col, w = _dev(torch, g.row_ptr, cuda_device), _dev(torch, g.col, cuda_device), _dev(torch, g.w, cuda_device)
    params = nps.Params(level=level, delta=delta, threshold=32, block_threshold=128, grid_threshold=1024)
    second = int(np.argsort(g.degrees(), kind="stable")[-7])
    for src in (g.source, second):  # two calls in a row on the shared scratch
        got = _solve(nps, torch, cuda_device, row, col, w, g, src, params)
        assert np.array_equal(got, oracle.sssp_heap(g.row_ptr, g.col, g.w, src))
        want, _ = nps.sssp(g, src, params)
        assert np.array_equal(got, want)


def test_noalloc_many_edges_use_larger_work_items(nps, oracle, cuda_device):
    """n at the limit and 16.8 M edges: the fixed table of grid-tier work items is
    only large enough because items grow to 2^7 chunks; checked against the oracle."""
    import torch
    g = nps.gen_uniform(NOALLOC_MAX_VERTICES, 128 * NOALLOC_MAX_VERTICES, 255, 5)
    row, col, w = _dev(torch, g.row_ptr, cuda_device), _dev(torch, g.col, cuda_device), _dev(torch, g.w, cuda_device)
    params = nps.Params(level=2, delta=0, threshold=32)
    want = oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)
    for _ in range(2):
        assert np.array_equal(_solve(nps, torch, cuda_device, row, col, w, g, 0, params), want)


def test_noalloc_exact_after_a_call_that_timed_out(nps, oracle, cuda_device):
    """A call whose bounded barrier wait runs out (test hook: an arrival that never
    comes) returns NPS_ERR_TIMEOUT and clears the shared stamps; the next call on
    the same scratch is exact."""
    import torch
    g = nps.gen_rmat(14, 16, seed=4)
    row, col, w = _dev(torch, g.row_ptr, cuda_device), _dev(torch, g.col, cuda_device), _dev(torch, g.w, cuda_device)
    out = torch.empty(g.n, dtype=torch.int32, device=cuda_device)
    rc, _ = _noalloc(nps, row, col, w, g.n, g.m, g.source, out,
                     nps.Params(level=2, delta=16, timeout_s=0.5, fault_inject_wait=True))
    assert rc == NPS_ERR_TIMEOUT
    got = _solve(nps, torch, cuda_device, row, col, w, g, g.source, nps.Params(level=2, delta=16))
    assert np.array_equal(got, oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source))


def test_noalloc_refuses_a_capturing_stream(nps, cuda_device):
    import torch
    g = nps.gen_uniform(1024, 8192, 100, 2)
    row, col, w = _dev(torch, g.row_ptr, cuda_device), _dev(torch, g.col, cuda_device), _dev(torch, g.w, cuda_device)
    out = torch.zeros(g.n, dtype=torch.int32, device=cuda_device)
    s = torch.cuda.Stream(cuda_device)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        out.add_(1)  # something to capture
        rc, _ = _noalloc(nps, row, col, w, g.n, g.m, 0, out, nps.Params(), stream=s.cuda_stream)
    assert rc == NPS_ERR_INVALID_ARG
    assert b"captured" in nps.lib.nps_last_error_string()
    del graph


def test_noalloc_rejects_graphs_beyond_its_scratch(nps, cuda_device):
    import torch
    n = NOALLOC_MAX_VERTICES + 1
    row = torch.zeros(n + 1, dtype=torch.int32, device=cuda_device)
    col = torch.zeros(4, dtype=torch.int32, device=cuda_device)
    out = torch.empty(n, dtype=torch.int32, device=cuda_device)
    rc, _ = _noalloc(nps, row, col, col, n, 0, 0, out, nps.Params())
    assert rc == NPS_ERR_CAPACITY  # before any device work
    assert b"at most 131072" in nps.lib.nps_last_error_string()
