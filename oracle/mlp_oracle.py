"""CPU fp32 reference of the policy MLP -- TEST INFRASTRUCTURE ONLY.

The checker for the training and inference kernels in
nested-parallelism_b200/csrc/nps_mlp.cu (the reference project has no learned
component, so this is the reference): 12 -> 32 (ReLU) -> 14 with the weight
matrices rounded to bf16 exactly as the kernels store them, fp32 arithmetic,
mean softmax cross-entropy of the delta head (logits 0..10) and the level head
(logits 11..13), each weighted by a per-sample weight over the weight sum.
"""
import numpy as np

IN, HID, OUT, ND, NL = 12, 32, 14, 11, 3


def bf16(a):
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def forward(w1, b1, w2, b2, X):
    W1, W2 = bf16(w1).astype(np.float64), bf16(w2).astype(np.float64)
    h = np.maximum(X.astype(np.float64) @ W1.T + b1, 0.0)
    return h, h @ W2.T + b2


def _ce(o, y):
    m = o.max(axis=1, keepdims=True)
    lz = np.log(np.exp(o - m).sum(axis=1, keepdims=True)) + m
    p = np.exp(o - lz)
    loss = (lz[:, 0] - o[np.arange(o.shape[0]), y])
    d = p.copy()
    d[np.arange(o.shape[0]), y] -= 1.0
    return loss, d


def loss_and_grads(w1, b1, w2, b2, X, yd, yl, wt=None):
    """Returns (loss, gw1, gb1, gw2, gb2) of the weighted mean two-head cross-entropy,
    gradients taken with respect to the bf16-rounded weights (what the kernels use)."""
    X = np.asarray(X, np.float64)
    B = X.shape[0]
    wt = np.ones(B) if wt is None else np.asarray(wt, np.float64)
    sc = wt / wt.sum()
    h, o = forward(w1, b1, w2, b2, X)
    d = np.zeros_like(o)
    loss = 0.0
    md = (yd >= 0) & (yd < ND)
    if md.any():
        l, g = _ce(o[md, :ND], yd[md])
        loss += float((l * sc[md]).sum())
        d[md, :ND] = g * sc[md, None]
    ml = (yl >= 0) & (yl < NL)
    if ml.any():
        l, g = _ce(o[ml, ND:], yl[ml])
        loss += float((l * sc[ml]).sum())
        d[ml, ND:] = g * sc[ml, None]
    gw2 = d.T @ h
    gb2 = d.sum(axis=0)
    dh = (d @ bf16(w2).astype(np.float64)) * (h > 0)
    gw1 = dh.T @ X
    gb1 = dh.sum(axis=0)
    return loss, gw1, gb1, gw2, gb2


def numeric_grad(fn, x, eps=1e-3):
    """Central finite differences of scalar fn at float64 array x."""
    g = np.zeros_like(x)
    flat = x.reshape(-1)
    gf = g.reshape(-1)
    for i in range(flat.size):
        old = flat[i]
        flat[i] = old + eps
        a = fn(x)
        flat[i] = old - eps
        b = fn(x)
        flat[i] = old
        gf[i] = (a - b) / (2 * eps)
    return g


def adam(master, grad, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * grad
    m2 = b2 * m2 + (1 - b2) * grad * grad
    mh = m1 / (1 - b1 ** step)
    vh = m2 / (1 - b2 ** step)
    return master - lr * mh / (np.sqrt(vh) + eps), m1, m2
