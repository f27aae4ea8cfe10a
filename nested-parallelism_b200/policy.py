"""Learned per-iteration policy for the persistent SSSP kernel.

A 2-layer MLP (12 features -> 32 ReLU -> 14 logits; bf16 weights, fp32
accumulation) picks, at every bucket advance, the next bucket width
delta = 2^k (k = 0..10) and, at every iteration, the consolidation level
(warp / block / grid).  Inference runs inside the persistent kernel
(policy_eval in csrc/nps_device.cuh); training runs on the GPU through the
forward / loss-backward / Adam kernels of csrc/nps_mlp.cu.  Device memory is
plain torch tensors; all arithmetic is in those kernels.

The 12 features (computed in-kernel after each iteration's barrier):
  0      log2(1 + next frontier size)
  1..8   fraction of the iteration's frontier in out-degree bins [4^k-1, 4^(k+1)-1)
  9      log2(1 + bucket advances so far)
  10     fraction of vertices reached
  11     improvements per scanned edge in the iteration

Delta-stepping is exact for any delta and any level, so the policy changes only
speed; the plain kernel remains the fallback (no weights loaded, or
Params.policy = POLICY_PLAIN) and distances are identical either way.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from ._native import NPS_MLP_HID as HID
from ._native import NPS_MLP_IN as IN
from ._native import NPS_MLP_OUT as OUT
from ._native import check, lib

N_DELTA = 11
N_LEVEL = 3


def bf16_round(a: np.ndarray) -> np.ndarray:
    """fp32 -> nearest-even bf16 -> fp32 (the rounding the kernels apply)."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    return (bf16_round(a).view(np.uint32) >> 16).astype(np.uint16)


@dataclass
class MLPWeights:
    w1: np.ndarray  # [HID, IN]
    b1: np.ndarray  # [HID]
    w2: np.ndarray  # [OUT, HID]
    b2: np.ndarray  # [OUT]
    mean: np.ndarray  # [IN] feature mean
    istd: np.ndarray  # [IN] 1 / feature std

    @staticmethod
    def init(seed: int = 0) -> "MLPWeights":
        rng = np.random.default_rng(seed)
        w1 = (rng.standard_normal((HID, IN)) * np.sqrt(2.0 / IN)).astype(np.float32)
        w2 = (rng.standard_normal((OUT, HID)) * np.sqrt(1.0 / HID)).astype(np.float32)
        return MLPWeights(w1, np.zeros(HID, np.float32), w2, np.zeros(OUT, np.float32),
                          np.zeros(IN, np.float32), np.ones(IN, np.float32))

    def save(self, path: str) -> None:
        np.savez(path, w1=self.w1, b1=self.b1, w2=self.w2, b2=self.b2, mean=self.mean, istd=self.istd)

    @staticmethod
    def load(path: str) -> "MLPWeights":
        z = np.load(path)
        return MLPWeights(*(np.asarray(z[k], np.float32) for k in ("w1", "b1", "w2", "b2", "mean", "istd")))


def load_into_kernel(wts: MLPWeights, device: int = 0) -> None:
    """Install the weights for Params(policy=POLICY_LEARNED) on `device`."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in
            (wts.w1, wts.b1, wts.w2, wts.b2, wts.mean, wts.istd)]
    check(lib.nps_policy_set_weights(device, *[a.ctypes.data for a in arrs]), "nps_policy_set_weights")


class GPUTrainer:
    """Adam training of the policy MLP on the GPU with the library's kernels."""

    def __init__(self, wts: MLPWeights, device, lr: float = 3e-3):
        import torch
        self.torch = torch
        self.dev = device
        self.lr = lr
        self.step_no = 0
        self.shapes = [(HID, IN), (HID,), (OUT, HID), (OUT,)]
        self.master = [torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(device)
                       for a in (wts.w1, wts.b1, wts.w2, wts.b2)]
        self.m1 = [torch.zeros_like(t) for t in self.master]
        self.m2 = [torch.zeros_like(t) for t in self.master]
        self.grad = [torch.zeros_like(t) for t in self.master]
        self.w1_bf = torch.from_numpy(bf16_bits(wts.w1).view(np.int16)).to(device)
        self.w2_bf = torch.from_numpy(bf16_bits(wts.w2).view(np.int16)).to(device)
        self.mean, self.istd = wts.mean.copy(), wts.istd.copy()
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def forward(self, X):
        t = self.torch
        X = t.as_tensor(X, dtype=t.float32, device=self.dev).contiguous()
        out = t.empty((X.shape[0], OUT), dtype=t.float32, device=self.dev)
        check(lib.nps_mlp_forward(self.w1_bf.data_ptr(), self.master[1].data_ptr(), self.w2_bf.data_ptr(),
                                  self.master[3].data_ptr(), X.data_ptr(), X.shape[0], out.data_ptr(),
                                  self._stream()), "nps_mlp_forward")
        return out

    def loss_backward(self, X, yd, yl, wt=None):
        """Zeroes and fills self.grad; returns the weighted mean loss (device)."""
        t = self.torch
        X = t.as_tensor(X, dtype=t.float32, device=self.dev).contiguous()
        yd = t.as_tensor(yd, dtype=t.int32, device=self.dev).contiguous()
        yl = t.as_tensor(yl, dtype=t.int32, device=self.dev).contiguous()
        wp = 0
        if wt is not None:
            wt = t.as_tensor(wt, dtype=t.float32, device=self.dev).contiguous()
            wp = wt.data_ptr()
        for g in self.grad:
            g.zero_()
        self.loss.zero_()
        check(lib.nps_mlp_loss_backward(self.w1_bf.data_ptr(), self.master[1].data_ptr(), self.w2_bf.data_ptr(),
                                        self.master[3].data_ptr(), X.data_ptr(), yd.data_ptr(), yl.data_ptr(),
                                        wp, X.shape[0], *[g.data_ptr() for g in self.grad],
                                        self.loss.data_ptr(), self._stream()), "nps_mlp_loss_backward")
        return self.loss

    def adam_step(self):
        self.step_no += 1
        bf = [self.w1_bf.data_ptr(), 0, self.w2_bf.data_ptr(), 0]
        for k in range(4):
            check(lib.nps_mlp_adam_step(self.master[k].data_ptr(), bf[k] or None, self.grad[k].data_ptr(),
                                        self.m1[k].data_ptr(), self.m2[k].data_ptr(), self.master[k].numel(),
                                        self.lr, 0.9, 0.999, 1e-8, self.step_no, self._stream()),
                  "nps_mlp_adam_step")

    def weights(self) -> MLPWeights:
        w1, b1, w2, b2 = (t.detach().cpu().numpy().copy() for t in self.master)
        return MLPWeights(w1, b1, w2, b2, self.mean.copy(), self.istd.copy())


def smoke_step(device) -> float:
    """One forward + backward + Adam step on a seeded random batch; returns the loss."""
    rng = np.random.default_rng(0)
    tr = GPUTrainer(MLPWeights.init(0), device)
    X = rng.standard_normal((512, IN)).astype(np.float32)
    yd = rng.integers(0, N_DELTA, 512)
    yl = rng.integers(0, N_LEVEL, 512)
    loss = float(tr.loss_backward(X, yd, yl).item())
    tr.adam_step()
    tr.torch.cuda.synchronize(device)
    assert np.isfinite(loss) and loss > 0
    return loss


# ---------------------------------------------------------------------------
# Training data from traces of plain runs.
#
# For every training graph the plain kernel runs once per fixed configuration
# (delta in DELTA_CHOICES x level in LEVEL_CHOICES, the other parameters those
# of the plain autotuned configuration) with tracing on.  A trace record holds
# the kernel's own feature vector after an iteration and the device time at
# which the iteration ended.  Each record is placed in a progress bin (reached
# vertices at that point over the reached total); the cost of a configuration
# in a bin is the device time of the iterations that start in it.  Every record
# of a graph is labelled with the configuration that is cheapest in the
# record's bin, weighted by how much that choice saves there against the median
# configuration.  The network so learns which bucket width and consolidation
# level pay off in which phase of a run.

DELTA_CHOICES = [1 << k for k in range(11)]
LEVEL_CHOICES = [0, 1, 2]
PROGRESS_BINS = np.array([0.0, 1e-3, 1e-2, 0.05, 0.2, 0.5, 0.8, 0.95, 0.99, 1.01])


def trace_run(dg, params, device: int = 0):
    """One traced run on a device-resident graph; returns (kernel_ms, records)."""
    import dataclasses as _dc
    from . import sssp_device, trace_read
    p = _dc.replace(params, trace=True, policy=0)
    st = sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p)
    return st.kernel_ms, trace_read(device)


def config_params(base, delta: int, level: int):
    import dataclasses as _dc
    return _dc.replace(base, delta=delta, level=level)


def _spread(c, p0, p1, dt):
    """Add an iteration's time dt to the progress bins its span [p0, p1) overlaps,
    in proportion to the overlap; a span without progress charges its own bin."""
    nb = len(PROGRESS_BINS) - 1
    if p1 <= p0 + 1e-12:
        b = int(np.searchsorted(PROGRESS_BINS, p0, side="right") - 1)
        c[min(max(b, 0), nb - 1)] += dt
        return
    lo = np.maximum(PROGRESS_BINS[:-1], p0)
    hi = np.minimum(PROGRESS_BINS[1:], p1)
    c += dt * np.clip(hi - lo, 0.0, None) / (p1 - p0)


def label_graph(runs):
    """runs: {(delta_idx, level_idx): (ms, records)} for one graph.
    Returns X [R, 12], yd [R], yl [R], wt [R] over all records of all runs."""
    final = max(recs[-1]["reached"] for _, recs in runs.values() if recs)
    nb = len(PROGRESS_BINS) - 1
    cost = {}
    rows = []
    for cfg, (ms, recs) in runs.items():
        c = np.zeros(nb)
        prev_t = 0.0
        prev_p = 0.0
        for r in recs:
            p1 = r["reached"] / max(final, 1)
            _spread(c, prev_p, p1, r["t_us"] - prev_t)
            prev_t = r["t_us"]
            prev_p = p1
            # the decision taken after this record shapes the iterations that start here
            b = min(max(int(np.searchsorted(PROGRESS_BINS, p1, side="right") - 1), 0), nb - 1)
            rows.append((cfg, b, r["feat"]))
        cost[cfg] = c
    cfgs = list(cost)
    C = np.stack([cost[k] for k in cfgs])  # [configs, bins]
    best = C.argmin(axis=0)
    gain = np.median(C, axis=0) - C.min(axis=0)
    X, yd, yl, wt = [], [], [], []
    for cfg, b, feat in rows:
        d_i, l_i = cfgs[best[b]]
        X.append(feat)
        yd.append(d_i)
        yl.append(l_i)
        wt.append(gain[b] + 1e-3)
    return (np.array(X, np.float32), np.array(yd, np.int64), np.array(yl, np.int64), np.array(wt, np.float32))


def train(X, yd, yl, wt, device, steps: int = 1500, lr: float = 3e-3, seed: int = 0, log_every: int = 0):
    """Fit the policy on the GPU with the library's kernels; returns (MLPWeights, losses)."""
    mean = X.mean(axis=0).astype(np.float32)
    std = X.std(axis=0).astype(np.float32)
    istd = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 0.0).astype(np.float32)
    Xn = ((X - mean) * istd).astype(np.float32)
    w = MLPWeights.init(seed)
    w.mean, w.istd = mean, istd
    tr = GPUTrainer(w, device, lr=lr)
    t = tr.torch
    Xd = t.as_tensor(Xn, device=device)
    ydd = t.as_tensor(yd.astype(np.int32), device=device)
    yld = t.as_tensor(yl.astype(np.int32), device=device)
    wtd = t.as_tensor(wt / wt.mean(), device=device)
    losses = []
    for i in range(steps):
        loss = tr.loss_backward(Xd, ydd, yld, wtd)
        tr.adam_step()
        if log_every and i % log_every == 0:
            losses.append(float(loss.item()))
    losses.append(float(tr.loss_backward(Xd, ydd, yld, wtd).item()))
    return tr.weights(), losses
