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
