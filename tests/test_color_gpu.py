"""Graph coloring on the GPU (nps_color, the graph-color application's
gclr_np_consolidate_gpu) against the oracle's closed form, which equals its
literal simulation of the reference's iterations (tests/test_color_cpu.py).
Colors are integers and the result does not depend on scheduling, so every case
is exact."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("threshold", [1, 8, 64, 1 << 20])
@pytest.mark.parametrize("kind", ["rmat16", "grid128", "uniform16k"])
def test_colors_match_the_oracle(nps, oracle, cuda_device, kind, threshold):
    g = {"rmat16": lambda: nps.gen_rmat(16, 16, seed=3), "grid128": lambda: nps.gen_grid(128, 128, 0.05, 10, 7),
         "uniform16k": lambda: nps.gen_uniform(16384, 131072, 100, 1)}[kind]()
    want, it = oracle.color(g.row_ptr, g.col)
    got, st = nps.color(g, nps.Params(threshold=threshold))
    assert np.array_equal(got, want)
    assert st.iterations == it and st.status == 0


def test_edge_cases(nps, oracle, cuda_device):
    for g in (nps.convertCSR(1, [], [], []), nps.convertCSR(5, [1, 2, 0, 0, 4], [2, 3, 1, 1, 0], [4, 5, 1, 1, 1]),
              nps.convertCSR(4, [3, 3, 3, 2, 3], [3, 2, 1, 0, 0], [1, 1, 1, 1, 1])):
        got, _ = nps.color(g)
        assert np.array_equal(got, oracle.color(g.row_ptr, g.col)[0])


def test_long_rows_and_deep_chains(nps, oracle, cuda_device):
    """A 300k-edge hub (scanned by a warp) and a 5000-vertex chain (5000 colors)."""
    n = 300001
    hub = nps.convertCSR(n, np.full(n - 1, n - 1), np.arange(n - 1), np.ones(n - 1, np.uint32))
    chain = nps.convertCSR(5000, np.arange(1, 5000), np.arange(4999), np.ones(4999, np.uint32))
    for g in (hub, chain):
        want, it = oracle.color(g.row_ptr, g.col)
        got, st = nps.color(g)
        assert np.array_equal(got, want) and st.iterations == it


def test_device_pointers_and_malformed_input(nps, oracle, cuda_device):
    import torch
    g = nps.gen_rmat(14, 8, seed=2)
    dev = cuda_device
    row = torch.from_numpy(g.row_ptr.view(np.int32)).to(dev)
    col = torch.from_numpy(g.col.view(np.int32)).to(dev)
    out = torch.empty(g.n, dtype=torch.int32, device=dev)
    st = nps.color_device(row, col, g.n, g.m, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle.color(g.row_ptr, g.col)[0]) and st.status == 0
    bad = g.col.copy()
    bad[10] = g.n + 5
    with pytest.raises(nps.NpsError) as ei:
        nps.color_device(row, torch.from_numpy(bad.view(np.int32)).to(dev), g.n, g.m, out)
    assert ei.value.status == 7


def test_bounded_barrier_wait_times_out_and_context_survives(nps, oracle, cuda_device):
    """The round kernel's grid barrier gives up after timeout_s: with the test hook its
    first barrier waits for an arrival that never comes; the call reports
    NPS_ERR_TIMEOUT and the next call on the same context is exact."""
    g = nps.gen_rmat(14, 8, seed=2)
    with pytest.raises(nps.NpsError) as ei:
        nps.color(g, nps.Params(fault_inject_wait=True, timeout_s=0.2))
    assert ei.value.status == 4
    got, st = nps.color(g)
    want, it = oracle.color(g.row_ptr, g.col)
    assert np.array_equal(got, want) and st.iterations == it
