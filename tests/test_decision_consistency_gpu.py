"""After each team barrier every CTA of the persistent kernel reads the shared
counters and must take the same decision (next light iteration, heavy-edge pass,
bucket advance or the end).  A faster CTA may already be in the next iteration
while a slower one decides, so the decision reads only counters of the finished
iteration that the next one leaves alone.  The settle list (light/heavy split) is
the case that once broke this: a bucket advance appends the far-pile vertices it
processes to the settle list, so a slow CTA that read the list's running tail could
take a heavy pass where the others advanced, and whole regions of the graph stayed
unreached with an OK status (about one run in ten of the case below).  The count
now comes from a per-iteration slot.

A 2048 x 2048 grid with delta 8 and the split runs about 260,000 iterations and
118,000 bucket advances per SSSP; every run must equal the CPU oracle
(apps/sssp/src/cpu/sssp.cpp:13-47)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_light_heavy_bucket_advances_stay_exact_over_many_runs(nps, oracle, cuda_device):
    import importlib
    at = importlib.import_module("nested-parallelism_b200.autotune")
    g = nps.gen_grid(2048, 2048, 0.05, 1000, 1)
    want = oracle.sssp_heap(g.row_ptr, g.col, g.w, 0)
    dg = at.to_device(g, 0, cuda_device)
    p = nps.Params(level=2, threshold=64, block_size=512, delta=8, light_heavy=True)
    for r in range(15):
        dg.dist.fill_(-1)
        st = nps.sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p)
        d = dg.dist.cpu().numpy().view(np.uint32)
        bad = int((d != want).sum())
        assert st.status == 0 and bad == 0, f"run {r}: {bad} mismatches, {st.iterations} iterations, {st.buckets} buckets"


def test_a_disagreement_is_reported_and_the_context_survives(nps, oracle, cuda_device):
    """The agreement check itself: with the test hook, CTA 1 adds another hash for the
    first decision (it still takes the same one), so every CTA finds the sum wrong one
    iteration later and the run ends with NPS_ERR_INTERNAL instead of a result.  No GPU
    fault is involved; the next call must be exact."""
    g = nps.gen_uniform(16384, 131072, 100, 1)
    with pytest.raises(nps.NpsError) as e:
        nps.sssp(g, 0, nps.Params(level=2, fault_inject_disagree=True))
    assert e.value.status == 9  # NPS_ERR_INTERNAL
    dist, st = nps.sssp(g, 0, nps.Params(level=2))
    assert st.status == 0
    assert np.array_equal(dist, oracle.sssp_heap(g.row_ptr, g.col, g.w, 0))
