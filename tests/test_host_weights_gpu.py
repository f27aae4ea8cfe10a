"""Host-pointer calls (SSSP_GPU's path: prepare_gpu() copies the CSR,
apps/sssp/src/gpu/sssp_wrapper.cu:58-149) move weights that fit in 8 or 16 bits
across PCIe packed and widen them on the device.  Whatever the width the weights
take (1, 2 or 4 bytes), including the boundaries 255/256 and 65535/65536, the
distances must equal the CPU oracle's, and a repeated call on the same context
(reusing the pinned staging) must too."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def base(nps):
    g = nps.gen_rmat(17, 16, seed=4)  # 1.94 M edges: above the packing minimum of 2^20
    assert g.m >= 1 << 20
    return g


@pytest.mark.parametrize("lo,hi", [(1, 255), (1, 256), (200, 65535), (1, 65536), (1, 1 << 29)])
def test_packed_weights_give_the_oracles_distances(nps, oracle, cuda_device, base, lo, hi):
    rng = np.random.default_rng(hi)
    w = rng.integers(lo, hi + 1, base.m, dtype=np.int64).astype(np.uint32)
    w[rng.integers(0, base.m)] = hi  # the largest weight is present
    g = dataclasses.replace(base, weightArray=w)
    want = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    for _ in range(2):
        dist, st = nps.sssp(g, g.source, nps.Params(level=2, threshold=32, block_size=512))
        assert st.status == 0
        assert np.array_equal(dist, want)


def test_small_graph_below_the_packing_minimum(nps, oracle, cuda_device):
    g = nps.gen_uniform(16384, 131072, 100, 1)
    dist, st = nps.sssp(g, 0, nps.Params(level=2))
    assert np.array_equal(dist, oracle.sssp_heap(g.row_ptr, g.col, g.w, 0))
