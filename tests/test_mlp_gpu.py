"""The policy MLP's bf16 training / inference kernels against the fp32 CPU oracle.

Tolerances: forward logits 1e-4 relative (fp32 sums in a different order);
loss and gradients 1e-3 relative (gradients are accumulated with fp32 atomics
in nondeterministic order); Adam 1e-5 relative.  The fused in-kernel policy must
take exactly the decisions the oracle's argmax gives for the features the
kernel recorded.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pol(nps):
    return importlib.import_module("nested-parallelism_b200.policy")


def _data(seed=0, B=4096):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((B, M.IN)).astype(np.float32)
    yd = rng.integers(0, M.ND, B)
    yl = rng.integers(-1, M.NL, B)
    wt = (rng.random(B) + 0.5).astype(np.float32)
    return X, yd, yl, wt


def test_forward_matches_oracle(nps, pol, cuda_device):
    w = pol.MLPWeights.init(3)
    w.b1[:] = np.linspace(-0.2, 0.2, M.HID)
    tr = pol.GPUTrainer(w, cuda_device)
    X, *_ = _data(1, 1000)
    got = tr.forward(X).cpu().numpy()
    _, want = M.forward(w.w1, w.b1, w.w2, w.b2, X)
    assert np.allclose(got, want, rtol=1e-4, atol=1e-5)


def test_loss_and_gradients_match_oracle(nps, pol, cuda_device):
    w = pol.MLPWeights.init(4)
    tr = pol.GPUTrainer(w, cuda_device)
    X, yd, yl, wt = _data(2)
    loss = float(tr.loss_backward(X, yd, yl, wt).item())
    want = M.loss_and_grads(w.w1, w.b1, w.w2, w.b2, X, yd, yl, wt)
    assert loss == pytest.approx(want[0], rel=1e-4)
    for g, ref in zip(tr.grad, want[1:]):
        g = g.cpu().numpy()
        assert np.allclose(g, ref, rtol=1e-3, atol=1e-6), np.abs(g - ref).max()


def test_adam_step_matches_oracle(nps, pol, cuda_device):
    w = pol.MLPWeights.init(5)
    tr = pol.GPUTrainer(w, cuda_device, lr=1e-2)
    X, yd, yl, wt = _data(3, 512)
    tr.loss_backward(X, yd, yl, wt)
    grads = [g.cpu().numpy().astype(np.float64) for g in tr.grad]
    tr.adam_step()
    for k, (m0, g) in enumerate(zip((w.w1, w.b1, w.w2, w.b2), grads)):
        want, _, _ = M.adam(m0.astype(np.float64), g, np.zeros_like(g), np.zeros_like(g), 1, 1e-2)
        assert np.allclose(tr.master[k].cpu().numpy(), want, rtol=1e-5, atol=1e-7)
    # the bf16 shadow copies are the rounded masters
    assert np.array_equal(tr.w1_bf.cpu().numpy().view(np.uint16), pol.bf16_bits(tr.master[0].cpu().numpy()))


def test_training_learns_a_separable_rule(nps, pol, cuda_device):
    rng = np.random.default_rng(7)
    X = rng.standard_normal((8192, M.IN)).astype(np.float32)
    yd = np.clip((X[:, 0] * 2 + 5).round(), 0, 10).astype(np.int64)
    yl = (X[:, 3] > 0).astype(np.int64) + (X[:, 4] > 1).astype(np.int64)
    tr = pol.GPUTrainer(pol.MLPWeights.init(0), cuda_device, lr=1e-2)
    first = float(tr.loss_backward(X, yd, yl).item())
    for _ in range(400):
        tr.loss_backward(X, yd, yl)
        tr.adam_step()
    last = float(tr.loss_backward(X, yd, yl).item())
    logits = tr.forward(X).cpu().numpy()
    acc_l = (logits[:, 11:].argmax(1) == yl).mean()
    assert last < 0.5 * first and acc_l > 0.9


def test_fused_policy_takes_the_oracle_decisions(nps, pol, cuda_device):
    g = nps.gen_rmat(15, 16, seed=12)
    w = pol.MLPWeights.init(9)
    w.mean[:] = 1.0
    w.istd[:] = 0.5
    pol.load_into_kernel(w, 0)
    p = nps.Params(policy=nps.POLICY_LEARNED, delta=16, trace=True, light_heavy=False, policy_min_edges=-1)
    d, st = nps.sssp(g, g.source, p)
    tr = nps.trace_read(0)  # the trace of the most recent call
    assert np.array_equal(d, nps.sssp(g, g.source, nps.Params())[0])  # exact regardless of the policy
    assert len(tr) == st.iterations and len(tr) > 2
    for a, b in zip(tr[:-1], tr[1:]):
        x = ((np.array(a["feat"], np.float64) - w.mean) * w.istd)[None, :]
        _, o = M.forward(w.w1, w.b1, w.w2, w.b2, x.astype(np.float32))
        assert (b["level"] & 0xFF) == int(o[0, 11:].argmax())


def test_fused_policy_widths_follow_the_oracle(nps, pol, cuda_device):
    """The first bucket's width comes from the start-state features and every
    advance's width from the features of the iteration before it."""
    g = nps.gen_rmat(14, 16, seed=21)
    w = pol.MLPWeights.init(17)
    w.b2[:11] = np.linspace(0.0, 0.5, 11)  # spread the width logits
    pol.load_into_kernel(w, 0)
    p = nps.Params(policy=nps.POLICY_LEARNED, trace=True, light_heavy=False, policy_min_edges=-1)
    d, st = nps.sssp(g, g.source, p)
    tr = nps.trace_read(0)

    def k_of(feat):
        x = ((np.asarray(feat, np.float64) - w.mean) * w.istd)[None, :]
        _, o = M.forward(w.w1, w.b1, w.w2, w.b2, x.astype(np.float32))
        return int(o[0, :11].argmax())

    assert tr[0]["delta"] == 1 << k_of(pol.start_features(g.n, int(g.row_ptr[g.source + 1] - g.row_ptr[g.source])))
    adv = 0
    for a, b in zip(tr[:-1], tr[1:]):
        if b["level"] & 0x200:
            assert b["delta"] == 1 << k_of(a["feat"])
            adv += 1
    assert adv == st.buckets
