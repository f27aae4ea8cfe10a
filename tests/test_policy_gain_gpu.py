"""What the trained policy gains, and that it never costs: the committed weights
(policy_weights.npz, trained by train_policy.py on R-MAT scales 16-20, seeds
0-99) against the same kernel without them on held-out R-MAT graphs of scales
16-22.  Distances must be identical to the oracle's.  Below NPS_POLICY_MIN_EDGES
edges the library runs the plain kernel even when the policy is asked for
(stats.policy_used); above it the policy must scan fewer edges and be faster.
Times are medians of several runs, compared with a margin, so that a shared GPU's
noise does not decide the outcome; the edge counts carry the rest."""
import dataclasses
import importlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "nested-parallelism_b200", "policy_weights.npz")
MIN_EDGES = 3_000_000  # NPS_POLICY_MIN_EDGES in include/nps.h


def _median_ms(nps, dg, p, reps=9):
    ts = [nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p).kernel_ms
          for _ in range(reps + 2)]
    return float(np.median(ts[2:]))


@pytest.fixture(scope="module")
def arms(nps):
    pol = importlib.import_module("nested-parallelism_b200.policy")
    pol.load_into_kernel(pol.MLPWeights.load(WEIGHTS), 0)
    with open(os.path.join(os.path.dirname(WEIGHTS), "policy_training.json")) as f:
        plain = nps.Params(**json.load(f)["plain_autotuned_on_scale20"])
    learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0)
    return plain, learned


@pytest.mark.parametrize("scale", [16, 17, 18, 19, 20, 21, 22])
def test_learned_policy_never_loses_and_gains_on_large_graphs(nps, oracle, cuda_device, arms, scale):
    at = importlib.import_module("nested-parallelism_b200.autotune")
    plain, learned = arms
    g = nps.gen_rmat(scale, 16, seed=1000 + scale)
    dg = at.to_device(g, device=cuda_device)
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    st_p = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, plain)
    assert np.array_equal(dg.dist.cpu().numpy().view(np.uint32), ref)
    st_l = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, learned)
    assert np.array_equal(dg.dist.cpu().numpy().view(np.uint32), ref)
    t_plain = _median_ms(nps, dg, plain)
    t_learned = _median_ms(nps, dg, learned)
    print(f"scale {scale}: m {g.m}, plain {t_plain:.3f} ms {st_p.edges_scanned} edges, learned {t_learned:.3f} ms "
          f"{st_l.edges_scanned} edges, policy used {st_l.policy_used}, learned/plain speed {t_plain / t_learned:.2f}")
    if g.m < MIN_EDGES:
        assert st_l.policy_used == nps.POLICY_PLAIN
        assert st_l.edges_scanned == pytest.approx(st_p.edges_scanned, rel=0.25)
    else:
        assert st_l.policy_used == nps.POLICY_LEARNED
        assert st_l.edges_scanned < 0.8 * st_p.edges_scanned
    assert t_learned <= 1.05 * t_plain  # never slower, up to timing noise
    if scale >= 20:
        assert t_learned < 0.9 * t_plain
