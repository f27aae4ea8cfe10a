"""What the trained policy gains: the committed weights (policy_weights.npz,
trained by train_policy.py on R-MAT scales 16-20, seeds 0-99) against the
same kernel without them on a held-out R-MAT graph.  Distances must be
identical (and the oracle's); the learned run must scan fewer edges and be
faster."""
import importlib
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "nested-parallelism_b200", "policy_weights.npz")


def _median_ms(nps, dg, p, reps=7):
    ts = [nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p).kernel_ms
          for _ in range(reps + 1)]
    return float(np.median(ts[1:]))


@pytest.mark.parametrize("scale,seed", [(20, 1000), (21, 1001)])
def test_learned_policy_beats_plain(nps, oracle, cuda_device, scale, seed):
    """Plain = the autotuned configuration the policy was trained with
    (policy_training.json); learned = the same with the policy on."""
    import dataclasses
    import json
    pol = importlib.import_module("nested-parallelism_b200.policy")
    at = importlib.import_module("nested-parallelism_b200.autotune")
    pol.load_into_kernel(pol.MLPWeights.load(WEIGHTS), 0)
    g = nps.gen_rmat(scale, 16, seed=seed)
    dg = at.to_device(g, device=cuda_device)
    with open(os.path.join(os.path.dirname(WEIGHTS), "policy_training.json")) as f:
        plain = nps.Params(**json.load(f)["plain_autotuned_on_scale20"])
    learned = dataclasses.replace(plain, policy=nps.POLICY_LEARNED, light_heavy=False, order_degree=0)
    t_plain = _median_ms(nps, dg, plain)
    st_p = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, plain)
    d_plain = dg.dist.cpu().numpy().view(np.uint32).copy()
    t_learned = _median_ms(nps, dg, learned)
    st_l = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, learned)
    d_learned = dg.dist.cpu().numpy().view(np.uint32).copy()
    ref = oracle.sssp_heap(g.row_ptr, g.col, g.w, g.source)
    assert np.array_equal(d_plain, ref) and np.array_equal(d_learned, ref)
    print(f"scale {scale}: plain {t_plain:.3f} ms {st_p.edges_scanned} edges, "
          f"learned {t_learned:.3f} ms {st_l.edges_scanned} edges, {st_l.buckets} buckets")
    assert st_l.edges_scanned < 0.8 * st_p.edges_scanned
    assert t_learned < 0.9 * t_plain

