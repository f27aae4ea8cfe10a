"""Learned per-iteration policy for the persistent SSSP kernel.

A 2-layer MLP (12 features -> 32 ReLU -> 14 logits; bf16 weights, fp32
accumulation) picks the width delta = 2^k (k = 0..10) of the first bucket
(from the start state) and of every bucket a bucket advance opens, and, at
every iteration, the consolidation level (warp / block / grid).  Inference runs
inside the persistent kernel (policy_eval_warp in csrc/nps_device.cuh); training
runs on the GPU through the
forward / loss-backward / Adam kernels of csrc/nps_mlp.cu.  Device memory is
plain torch tensors; all arithmetic is in those kernels.

The 12 features (computed in-kernel after each iteration's barrier):
  0      log2(1 + next frontier size)
  1..8   fraction of the iteration's frontier in out-degree bins [4^k-1, 4^(k+1)-1)
  9      log2(1 + bucket advances so far)
  10     fraction of vertices reached
  11     improvements per scanned edge in the iteration

Delta-stepping is exact for any delta and any level, so the policy changes only
speed; the plain kernel (Params.policy = POLICY_PLAIN, the default) remains the
fallback and the check of every learned result, and distances are identical
either way.  A learned call
on a device without weights loaded is an error, not a silent fallback.
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
# Training data: imitation of the best bucket schedule of the plain kernel.
#
# The plain kernel runs a fixed bucket width, or a scripted per-bucket width
# schedule (Params.delta_schedule).  For every training graph a teacher search
# times the plain kernel under each candidate schedule (a few narrow leading
# buckets, then wide ones) and under each consolidation level, keeps the
# fastest, and runs it once more with tracing on.  Every trace record holds the
# kernel's own feature vector after an iteration; the record that precedes a
# bucket advance is labelled with the log2 width the schedule gave the bucket
# that advance opened, and every record with the best level.  The start state
# (before the first iteration) is labelled with the first bucket's width.  The
# network so learns, from frontier statistics alone, when narrow buckets pay
# for their extra iterations and when the run should go unordered.

LEVEL_CHOICES = [0, 1, 2]
LEADING_K = (0, 1, 2, 3)   # log2 widths tried for the leading buckets
REST_K = (8, 10)           # log2 width of every later bucket


def candidate_schedules(max_lead: int = 4):
    """(leading exponents, rest exponent) pairs: non-decreasing leading widths,
    1..max_lead of them, then a wide remainder; plus the wide width from the
    start (the plain kernel's unordered behaviour on these graphs)."""
    import itertools
    out = [((r,), r) for r in REST_K]
    for n in range(1, max_lead + 1):
        for lead in itertools.combinations_with_replacement(LEADING_K, n):
            for r in REST_K:
                out.append((tuple(lead), r))
    return out


def schedule_params(base, lead, rest, level=None):
    import dataclasses as _dc
    from . import delta_schedule
    kw = dict(delta_schedule=delta_schedule(list(lead), rest), policy=0, light_heavy=False, order_degree=0)
    if level is not None:
        kw["level"] = level
    return _dc.replace(base, **kw)


def _time(dg, params, reps: int = 3) -> float:
    from . import sssp_device
    sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, params)  # warm-up
    ts = [sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, params).kernel_ms
          for _ in range(reps)]
    return float(np.median(ts))


LEVEL_MARGIN = 0.05  # another level must beat the plain configuration's by 5 % to become the label


def teacher_search(dg, base, schedules, reps: int = 3):
    """Fastest (schedule, level) for one device graph.  Returns
    (best_ms, (lead, rest), level, {schedule: ms}).  The level label stays the plain
    configuration's unless another level is faster by LEVEL_MARGIN: level timings
    within a few percent are noise, and labels that flip between them teach the
    network nothing."""
    times = {}
    for lead, rest in schedules:
        times[(lead, rest)] = _time(dg, schedule_params(base, lead, rest), reps)
    best = min(times, key=times.get)
    lv_ms = {lv: _time(dg, schedule_params(base, best[0], best[1], lv), reps) for lv in LEVEL_CHOICES}
    level = base.level if base.level in lv_ms else min(lv_ms, key=lv_ms.get)
    fastest = min(lv_ms, key=lv_ms.get)
    if lv_ms[fastest] < (1.0 - LEVEL_MARGIN) * lv_ms[level]:
        level = fastest
    return lv_ms[level], best, level, times


def degree_bin(d: int) -> int:
    """Out-degree bin of the frontier histogram: [4^k - 1, 4^(k+1) - 1), last bin open."""
    return min(((int(d) + 1).bit_length() - 1) >> 1, 7)


def start_features(n: int, source_degree: int = None, frontier: int = 1) -> np.ndarray:
    """The start-state features the kernel evaluates before its first iteration.
    A single-source start reports the frontier that fills the first bucket, the
    source's out-neighbours: log2(1 + out-degree) and the source's degree bin; a
    start from a state reports log2(1 + frontier) and no histogram.  1/n reached."""
    f = np.zeros(IN, np.float32)
    f[0] = np.log2(1.0 + frontier)
    if source_degree is not None and frontier == 1:
        f[0] = np.log2(1.0 + int(source_degree))
        f[1 + degree_bin(int(source_degree))] = 1.0
    f[10] = 1.0 / n
    return f


def trace_schedule(dg, base, lead, rest, level, device: int = 0):
    """One traced plain run under a schedule; returns its trace records."""
    import dataclasses as _dc
    from . import sssp_device, trace_read
    p = _dc.replace(schedule_params(base, lead, rest, level), trace=True)
    sssp_device(dg.row_ptr, dg.col, dg.w, dg.n, dg.m, dg.src, dg.dist, p)
    return trace_read(device)


def label_trace(recs, n: int, lead, level: int, weight: float = 1.0, source_degree: int = None):
    """X [R+1, 12], yd [R+1] (-1 where no bucket decision follows), yl, wt."""
    X = [start_features(n, source_degree)]
    yd = [int(lead[0])]
    for i, r in enumerate(recs):
        X.append(np.asarray(r["feat"], np.float32))
        nxt = recs[i + 1] if i + 1 < len(recs) else None
        if nxt is not None and (nxt["level"] & 0x200) and nxt["delta"] > 0:
            yd.append(int(np.log2(nxt["delta"])))
        else:
            yd.append(-1)
    R = len(X)
    return (np.stack(X).astype(np.float32), np.array(yd, np.int64), np.full(R, level, np.int64),
            np.full(R, weight, np.float32))


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
