"""The MLP oracle's analytic gradients against central finite differences (CPU).

Weights are kept exactly representable in bf16 so that the finite differences
and the bf16 rounding inside the oracle agree."""
import numpy as np

import mlp_oracle as M


def _setup(seed=0, B=64):
    rng = np.random.default_rng(seed)
    w1 = M.bf16(rng.standard_normal((M.HID, M.IN)) * 0.4).astype(np.float64)
    w2 = M.bf16(rng.standard_normal((M.OUT, M.HID)) * 0.3).astype(np.float64)
    b1 = rng.standard_normal(M.HID) * 0.1
    b2 = rng.standard_normal(M.OUT) * 0.1
    X = rng.standard_normal((B, M.IN))
    yd = rng.integers(0, M.ND, B)
    yl = rng.integers(-1, M.NL, B)  # -1 drops the level head for some samples
    wt = rng.random(B) + 0.5
    return w1, b1, w2, b2, X, yd, yl, wt


def test_bias_gradients_match_finite_differences():
    w1, b1, w2, b2, X, yd, yl, wt = _setup()
    _, _, gb1, _, gb2 = M.loss_and_grads(w1, b1, w2, b2, X, yd, yl, wt)
    ng1 = M.numeric_grad(lambda b: M.loss_and_grads(w1, b, w2, b2, X, yd, yl, wt)[0], b1.copy(), 1e-5)
    ng2 = M.numeric_grad(lambda b: M.loss_and_grads(w1, b1, w2, b, X, yd, yl, wt)[0], b2.copy(), 1e-5)
    assert np.allclose(gb1, ng1, atol=1e-7, rtol=1e-4)
    assert np.allclose(gb2, ng2, atol=1e-7, rtol=1e-4)


def test_weight_gradients_match_finite_differences():
    # bf16 rounding makes the loss piecewise constant in the weights at bf16 resolution,
    # so the check perturbs inputs of an equivalent fp32 model: with weights already in
    # bf16, d loss / d W equals the gradient of the unrounded model, checked here on X
    # (linear in W1) through the identity dL/dW1 = dh^T X and a finite-difference check
    # of dL/dX, which shares dh.
    w1, b1, w2, b2, X, yd, yl, wt = _setup(1, 16)
    loss, gw1, _, gw2, _ = M.loss_and_grads(w1, b1, w2, b2, X, yd, yl, wt)
    # dL/dX from the same backward quantities
    h, o = M.forward(w1, b1, w2, b2, X)
    sc = wt / wt.sum()
    d = np.zeros_like(o)
    d[:, :M.ND] = M._ce(o[:, :M.ND], yd)[1] * sc[:, None]
    ml = yl >= 0
    d[ml, M.ND:] = M._ce(o[ml, M.ND:], yl[ml])[1] * sc[ml, None]
    dh = (d @ w2) * (h > 0)
    gX = dh @ w1
    ngX = M.numeric_grad(lambda x: M.loss_and_grads(w1, b1, w2, b2, x, yd, yl, wt)[0], X.copy(), 1e-6)
    assert np.allclose(gX, ngX, atol=1e-7, rtol=1e-3)
    assert np.allclose(gw1, dh.T @ X) and np.allclose(gw2, d.T @ h)


def test_adam_reference_moves_against_the_gradient():
    x = np.array([1.0, -2.0, 3.0])
    g = np.array([0.5, -0.5, 0.0])
    y, m1, m2 = M.adam(x, g, np.zeros(3), np.zeros(3), 1, 0.1)
    assert y[0] < x[0] and y[1] > x[1] and y[2] == x[2]
