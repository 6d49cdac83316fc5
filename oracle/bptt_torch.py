"""TEST INFRASTRUCTURE ONLY: the differentiable mode's dynamics unrolled in
PyTorch, differentiated by autograd.

This is the checker of the hand-written BPTT adjoint
(nemosim_b200/csrc/bptt.cu): run in float64 it is the FP64 oracle, in
float32 on the GPU it is the "PyTorch autograd" speed baseline.  The model is
the one documented in nemosim_b200/bptt.py; every operation below mirrors a
line of the native forward pass.
"""
from __future__ import annotations

import math

import torch


class _SpikeFn(torch.autograd.Function):
    """Heaviside forward, fast-sigmoid derivative k / (2 (1 + k|x|)^2) backward."""

    @staticmethod
    def forward(ctx, x):
        ctx.save_for_backward(x)
        return (x >= 0).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        q = 1.0 + 10.0 * x.abs()
        return g * (0.5 * 10.0 / (q * q))


def _smooth_spike(x):
    return 0.5 * (1.0 + 10.0 * x / (1.0 + 10.0 * x.abs()))


class Structure:
    """Synapses grouped by delay, for vectorised delayed input."""

    def __init__(self, source, target, delay, neurons: int, device):
        self.neurons = neurons
        self.groups = []
        src = torch.as_tensor(source.astype("int64"), device=device)
        tgt = torch.as_tensor(target.astype("int64"), device=device)
        dly = torch.as_tensor(delay.astype("int64"), device=device)
        self.max_delay = int(dly.max().item()) if len(dly) else 0
        for dl in range(1, self.max_delay + 1):
            idx = torch.nonzero(dly == dl).flatten()
            if len(idx):
                self.groups.append((dl, idx, src[idx], tgt[idx]))


def loss(W, a, b, c, d, noise, target, structure: Structure, readout: int, smooth: bool = False):
    """Loss of the unrolled dynamics; W [M], a b c d [N], noise [T,B,N],
    target [T,B,R]."""
    T, B, N = noise.shape
    dtype = noise.dtype
    spike = _smooth_spike if smooth else _SpikeFn.apply
    alpha = math.exp(-1.0 / 20.0)
    v = torch.full((B, N), -65.0, dtype=dtype, device=noise.device)
    u = b.unsqueeze(0) * v
    r = torch.zeros((B, readout), dtype=dtype, device=noise.device)
    hist = []
    total = torch.zeros((), dtype=dtype, device=noise.device)
    for t in range(T):
        syn = torch.zeros((B, N), dtype=dtype, device=noise.device)
        for dl, idx, src, tgt in structure.groups:
            if t >= dl:
                syn = syn.index_add(1, tgt, W[idx].unsqueeze(0) * hist[t - dl][:, src])
        I = syn + noise[t]
        S = torch.zeros((B, N), dtype=dtype, device=noise.device)
        for _ in range(4):
            v1 = v + 0.25 * (0.04 * v * v + 5.0 * v + 140.0 - u + I)
            u1 = u + 0.25 * a * (b * v1 - u)
            s = spike(v1 - 30.0)
            v = v1 + s * (c - v1)
            u = u1 + s * d
            S = S + s
        hist.append(S)
        r = alpha * r + S[:, :readout]
        total = total + ((r - target[t]) ** 2).sum()
    return total / (T * readout * B)
