"""Parity at the full sizes of the power-law and high-diameter configurations.

R-MAT scale 20 (1,048,576 vertices, edge factor 16, deduplicated) from the
highest out-degree vertex, and the 4096 x 4096 grid with 5 % of its edge pairs
dropped (16,777,216 vertices, about 63.7 M edges) from the corner (0, 0).  These
are the sizes at which the reference's fixed 10.24 M-entry queue and buffer
overflow (apps/sssp/src/gpu/sssp_wrapper.cu:496-502, sssp_kernel.cu:354-356 and
:414-431); here every queue is sized from n and m, and the distances must equal
the CPU oracle's Dijkstra bit for bit at the warp, block and grid consolidation
levels and under the learned policy.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(os.path.dirname(HERE), "nested-parallelism_b200", "policy_weights.npz")


@pytest.fixture(scope="module")
def rmat20(nps, oracle):
    g = nps.gen_rmat(20, 16, seed=1)
    return g, oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)


@pytest.fixture(scope="module")
def grid4096(nps, oracle):
    g = nps.gen_grid(4096, 4096, 0.05, 1000, 1)
    assert g.source == 0
    return g, oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)


@pytest.fixture(scope="module")
def learned_weights(nps, cuda_device):
    import importlib
    pol = importlib.import_module("nested-parallelism_b200.policy")
    pol.load_into_kernel(pol.MLPWeights.load(WEIGHTS), 0)
    return True


def _check(nps, g, want, params):
    dist, st = nps.sssp(g, g.source, params)
    bad = np.nonzero(dist != want)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}"
    assert st.status == 0
    return st


@pytest.mark.parametrize("level", [0, 1, 2])
@pytest.mark.parametrize("delta", [0, 64])
def test_rmat20_levels(nps, cuda_device, rmat20, level, delta):
    g, want = rmat20
    assert g.n == 1 << 20 and g.m > 10_000_000
    _check(nps, g, want, nps.Params(level=level, delta=delta, threshold=64, block_size=512))


def test_rmat20_learned_policy(nps, cuda_device, rmat20, learned_weights):
    g, want = rmat20
    st = _check(nps, g, want, nps.Params(level=2, threshold=32, block_size=512, policy=nps.POLICY_LEARNED,
                                         light_heavy=False))
    assert st.buckets >= 1


@pytest.mark.parametrize("level", [0, 1, 2])
def test_grid4096_levels(nps, cuda_device, grid4096, level):
    g, want = grid4096
    assert g.n == 4096 * 4096 and 60_000_000 < g.m < 67_092_480
    st = _check(nps, g, want, nps.Params(level=level, delta=4096, threshold=64, block_size=256))
    assert st.buckets > 100  # a long bucket sequence with small frontiers


def test_grid4096_learned_policy(nps, cuda_device, grid4096, learned_weights):
    g, want = grid4096
    _check(nps, g, want, nps.Params(level=2, threshold=32, block_size=512, policy=nps.POLICY_LEARNED,
                                    light_heavy=False, timeout_s=30.0))
