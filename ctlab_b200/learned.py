"""Learned warm start for OS-SART: a 2.5D residual CNN trained and run with
the library's own tensor-core kernels (ctlab_cnn_*, include/ctlab_b200.h).

Network, one z slice at a time: 5 input channels (the slice and two
neighbours each side of a scaled OS-SART image), conv 5->64 + ReLU,
6 x (conv 64->64 + ReLU), conv 64->1, output = centre slice + last conv.
Weights and activations are BF16 (NHWC), accumulation FP32, master weights
and Adam moments FP32.  torch tensors only hold device memory.

Training pairs come from the method itself: the 2-iteration OS-SART image
(input) and the 30-iteration image (target) of the same noisy projections.
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import check, load

LAYERS = [(16, 64)] + [(64, 64)] * 6 + [(64, 16)]  # (ci, co) padded channel counts
EPI_RELU, EPI_MASK, EPI_RESIDUAL = 0, 1, 2


def _p(t):
    return None if t is None else t.data_ptr()


class WarmStartNet:
    """The CNN's parameters, optimizer state and activations on one device."""

    def __init__(self, seed: int = 0, device: str = "cuda"):
        import torch
        self.torch = torch
        self.lib = load()
        self.dev = device
        g = np.random.default_rng(seed)
        self.params, self.m, self.v, self.grad, self.wf, self.wt = [], [], [], [], [], []
        for li, (ci, co) in enumerate(LAYERS):
            ci_real = 5 if li == 0 else ci
            co_real = 1 if li == len(LAYERS) - 1 else co
            w = np.zeros((co, 9, ci), np.float32)
            std = math.sqrt(2.0 / (9 * ci_real)) * (0.1 if co_real == 1 else 1.0)
            w[:co_real, :, :ci_real] = g.normal(0.0, std, (co_real, 9, ci_real))
            flat = np.concatenate([w.ravel(), np.zeros(co, np.float32)])
            self.params.append(torch.from_numpy(flat).to(device))
            for lst in (self.m, self.v, self.grad):
                lst.append(torch.zeros_like(self.params[-1]))
            self.wf.append(torch.empty(co * 9 * ci, dtype=torch.bfloat16, device=device))
            self.wt.append(torch.empty(co * 9 * ci, dtype=torch.bfloat16, device=device))
            self._sync_bf16(li)
        self.step_count = 0
        self.acts = []

    def _sync_bf16(self, li):
        ci, co = LAYERS[li]
        w = self.params[li][: co * 9 * ci].view(co, 9, ci)
        self.wf[li].copy_(w.reshape(-1).to(self.torch.bfloat16))
        self.wt[li].copy_(w.flip(1).permute(2, 1, 0).contiguous().reshape(-1).to(self.torch.bfloat16))

    def bias(self, li):
        ci, co = LAYERS[li]
        return self.params[li][co * 9 * ci:]

    # ------------------------------------------------------------------
    def forward(self, inp, center):
        """inp: bf16 [B,H,W,16]; center: f32 [B,H,W] -> prediction f32 [B,H,W]."""
        torch = self.torch
        B, H, W, _ = inp.shape
        x = inp
        self.acts = [inp]
        for li, (ci, co) in enumerate(LAYERS[:-1]):
            out = torch.empty((B, H, W, co), dtype=torch.bfloat16, device=self.dev)
            check(self.lib.ctlab_cnn_conv(_p(x), ci, _p(self.wf[li]), _p(self.bias(li)), co, B, H, W, EPI_RELU,
                                          _p(out), None, None, None, None))
            self.acts.append(out)
            x = out
        pred = torch.empty((B, H, W), dtype=torch.float32, device=self.dev)
        li = len(LAYERS) - 1
        ci, co = LAYERS[li]
        check(self.lib.ctlab_cnn_conv(_p(x), ci, _p(self.wf[li]), _p(self.bias(li)), co, B, H, W, EPI_RESIDUAL,
                                      None, None, _p(pred), _p(center), None))
        return pred

    def backward(self, pred, target):
        """Accumulates parameter gradients of the MSE loss; returns the loss."""
        torch = self.torch
        B, H, W = pred.shape
        n = B * H * W
        g = torch.empty((B, H, W, 16), dtype=torch.bfloat16, device=self.dev)
        acc = torch.zeros(1, dtype=torch.float64, device=self.dev)
        check(self.lib.ctlab_cnn_loss_grad(_p(pred), _p(target), n, _p(g), _p(acc), None))
        dpre = g
        for li in range(len(LAYERS) - 1, -1, -1):
            ci, co = LAYERS[li]
            a_in = self.acts[li]
            gw = self.grad[li]
            check(self.lib.ctlab_cnn_wgrad(_p(dpre), co, _p(a_in), ci, B, H, W, _p(gw), _p(gw[co * 9 * ci:]), None))
            if li == 0:
                break
            # data gradient through this layer, masked by the previous ReLU
            d_in = torch.empty((B, H, W, ci), dtype=torch.bfloat16, device=self.dev)
            check(self.lib.ctlab_cnn_conv(_p(dpre), co, _p(self.wt[li]), None, ci, B, H, W, EPI_MASK, _p(d_in),
                                          _p(a_in), None, None, None))
            dpre = d_in
        return float(acc.item()) / n

    def step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.step_count += 1
        for li, (ci, co) in enumerate(LAYERS):
            check(self.lib.ctlab_cnn_adam(_p(self.params[li]), _p(self.m[li]), _p(self.v[li]), _p(self.grad[li]), co,
                                          ci, lr, b1, b2, eps, self.step_count, _p(self.wf[li]), _p(self.wt[li]),
                                          None))

    # ------------------------------------------------------------------
    def pack(self, vol, zs, scale, target=None):
        """Network inputs (and targets) for slices zs of device volumes [YN][XN][ZN]."""
        torch = self.torch
        YN, XN, ZN = vol.shape
        z = torch.as_tensor(np.asarray(zs, np.int32), device=self.dev)
        nb = len(zs)
        inp = torch.empty((nb, YN, XN, 16), dtype=torch.bfloat16, device=self.dev)
        center = torch.empty((nb, YN, XN), dtype=torch.float32, device=self.dev)
        tgt = torch.empty((nb, YN, XN), dtype=torch.float32, device=self.dev) if target is not None else None
        check(self.lib.ctlab_cnn_pack(_p(vol), XN, YN, ZN, _p(z), nb, scale, _p(inp), _p(center), _p(tgt),
                                      _p(target), None))
        return inp, center, tgt

    def train_step(self, vol_in, vol_target, zs, scale, lr):
        inp, center, tgt = self.pack(vol_in, zs, scale, vol_target)
        pred = self.forward(inp, center)
        loss = self.backward(pred, tgt)
        self.step(lr)
        return loss

    def check_kernels(self):
        """Raises if a convolution gave up waiting for its tensor-core MMAs
        since the last check (synchronises the current stream)."""
        check(self.lib.ctlab_cnn_check(None))

    def predict_volume(self, vol_in, scale, out, batch: int = 16):
        """Runs the network over every z slice of vol_in into out (both [YN][XN][ZN])."""
        torch = self.torch
        YN, XN, ZN = vol_in.shape
        for z0 in range(0, ZN, batch):
            zs = list(range(z0, min(ZN, z0 + batch)))
            inp, center, _ = self.pack(vol_in, zs, scale)
            pred = self.forward(inp, center)
            z = torch.as_tensor(np.asarray(zs, np.int32), device=self.dev)
            check(self.lib.ctlab_cnn_unpack(_p(pred), XN, YN, ZN, _p(z), len(zs), scale, _p(out), None))
        self.acts = []
        return out
