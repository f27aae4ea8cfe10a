"""nps_sssp_noalloc, the entry point that allocates nothing, against nps_sssp.

Some callers of this library cannot allocate device memory at the moment they
ask for shortest paths: a stream being captured into a CUDA graph in global
mode (cudaMalloc fails there), a service that has reserved all device memory in
its own pool, a host that forbids allocator calls from its callbacks.
nps_sssp_noalloc serves them from a static device array sized for graphs of up
to NPS_NOALLOC_MAX_VERTICES vertices.  Its distances must equal those of the
regular entry point bit for bit (integer distances: zero tolerance), and must
stay equal on a second call in a row, since calls reuse the same array.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_VERTICES = 131072  # NPS_NOALLOC_MAX_VERTICES in include/nps.h


def _dev(torch, a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)


def _noalloc(nps, row, col, w, n, m, src, out, params):
    from importlib import import_module
    native = import_module("nested-parallelism_b200._native")
    p = params.to_c(device_ptrs=True)
    st = native.nps_stats()
    rc = nps.lib.nps_sssp_noalloc(row.data_ptr(), col.data_ptr(), w.data_ptr(), n, m, src, out.data_ptr(),
                                  C.byref(p), C.byref(st))
    return rc, st


@pytest.mark.parametrize("level,delta", [(2, 32), (1, 0), (3, 64)])
def test_noalloc_matches_nps_sssp_on_two_calls(nps, cuda_device, level, delta):
    import torch
    g = nps.gen_rmat(16, 16, seed=21)  # 65,536 vertices, inside the limit
    assert g.n <= NOALLOC_MAX_VERTICES
    row, col, w = _dev(torch, g.row_ptr, cuda_device), _dev(torch, g.col, cuda_device), _dev(torch, g.w, cuda_device)
    params = nps.Params(level=level, delta=delta, threshold=32, block_threshold=128, grid_threshold=1024)
    second = int(np.argsort(g.degrees(), kind="stable")[-7])
    for src in (g.source, second):  # two calls in a row on the shared scratch
        want, _ = nps.sssp(g, src, params)
        out = torch.full((g.n,), -1, dtype=torch.int32, device=cuda_device)
        rc, st = _noalloc(nps, row, col, w, g.n, g.m, src, out, params)
        assert rc == 0, nps.lib.nps_last_error_string().decode()
        assert st.status == 0 and st.iterations > 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)


def test_noalloc_rejects_graphs_beyond_its_scratch(nps, cuda_device):
    import torch
    n = NOALLOC_MAX_VERTICES + 1
    row = torch.zeros(n + 1, dtype=torch.int32, device=cuda_device)
    col = torch.zeros(4, dtype=torch.int32, device=cuda_device)
    out = torch.empty(n, dtype=torch.int32, device=cuda_device)
    rc, _ = _noalloc(nps, row, col, col, n, 0, 0, out, nps.Params())
    assert rc == 3  # NPS_ERR_CAPACITY, before any device work
    assert b"at most 131072" in nps.lib.nps_last_error_string()
