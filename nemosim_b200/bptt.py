"""Differentiable float32 mode: the hand-written BPTT adjoint of the native
library (nemosim_b200/csrc/bptt.cu) behind a ``torch.autograd.Function``.
Weights, parameters, noise, targets and gradients are float32 tensors.  The
neuron state, trajectories and adjoints are float64 by default
(``state_dtype=torch.float64``): the gradient of a spiking network amplifies
rounding, and at 4096 neurons x 500 ms x 16 trials a float32 evaluation of
the hard-threshold dynamics fires different spikes than a float64 one (its
gradient, like PyTorch's float32 autograd of the same model, is off by a
factor of about 100), while float64 state matches the float64 evaluation to
about 3e-8 at the same speed.  ``state_dtype=torch.float32`` keeps float32
state.

The model: Izhikevich neurons with 4 Euler sub-steps per ms (as
src/nemo/cpu/plugins/Izhikevich.cpp), a reset after every sub-step, delayed
float32 synapses, Gaussian input noise, and a loss on the exponentially
filtered (tau = 20 ms) spike trains of the readout neurons.  The threshold is
the Heaviside step in the forward pass and a fast sigmoid (slope 10) in the
backward pass; ``smooth=True`` uses the fast sigmoid in the forward pass too,
which makes the loss differentiable so that finite differences can check the
adjoint.

    net = DifferentiableNetwork.random(4096, 200, max_delay=10, seed=1)
    model = net.model(trials=16, ms=500, readout=256, checkpoint_ms=50)
    W, a, b = net.tensors(device)            # leaf tensors with requires_grad
    loss = model.loss(W, a, b, noise, target)
    loss.backward()                          # W.grad, a.grad, b.grad
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import NemoError, _check, lib


@dataclass
class DifferentiableNetwork:
    """Structure and initial parameters of a differentiable network: synapses
    ordered by source (weight w[e] belongs to synapse e)."""
    source: np.ndarray
    target: np.ndarray
    delay: np.ndarray
    weight: np.ndarray
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray
    d: np.ndarray

    @property
    def neurons(self) -> int:
        return len(self.a)

    @staticmethod
    def random(neurons: int, fanout: int, max_delay: int = 10, seed: int = 0, exc_fraction: float = 0.8):
        """80/20 excitatory/inhibitory Izhikevich neurons (the parameter
        distributions of src/examples/random.cpp), `fanout` outgoing synapses
        per neuron to uniform random targets, weights N(0, 0.5/sqrt(fanout)),
        delays uniform in 1..max_delay."""
        rng = np.random.default_rng(seed)
        n_exc = int(neurons * exc_fraction)
        exc = np.arange(neurons) < n_exc
        r1 = rng.random(neurons).astype(np.float32)
        r2 = rng.random(neurons).astype(np.float32)
        a = np.where(exc, 0.02, 0.02 + 0.08 * r1).astype(np.float32)
        b = np.where(exc, 0.2, 0.25 - 0.05 * r2).astype(np.float32)
        c = np.where(exc, -65.0 + 15.0 * r1 * r1, -65.0).astype(np.float32)
        d = np.where(exc, 8.0 - 6.0 * r2 * r2, 2.0).astype(np.float32)
        src = np.repeat(np.arange(neurons, dtype=np.uint32), fanout)
        tgt = rng.integers(0, neurons, size=len(src), dtype=np.uint32)
        dly = rng.integers(1, max_delay + 1, size=len(src), dtype=np.uint32)
        w = rng.normal(0.0, 0.5 / np.sqrt(fanout), size=len(src)).astype(np.float32)
        return DifferentiableNetwork(src, tgt, dly, w, a, b, c, d)

    def tensors(self, device, dtype=torch.float32, requires_grad=True):
        """(W, a, b) as leaf tensors and (c, d) as constants."""
        W = torch.tensor(self.weight, device=device, dtype=dtype, requires_grad=requires_grad)
        a = torch.tensor(self.a, device=device, dtype=dtype, requires_grad=requires_grad)
        b = torch.tensor(self.b, device=device, dtype=dtype, requires_grad=requires_grad)
        return W, a, b

    def constants(self, device, dtype=torch.float32):
        return (torch.tensor(self.c, device=device, dtype=dtype), torch.tensor(self.d, device=device, dtype=dtype))

    def model(self, trials: int, ms: int, readout: int, checkpoint_ms: int = 50, smooth: bool = False,
              device: int | None = None, state_dtype: torch.dtype = torch.float64) -> "BpttModel":
        """``state_dtype=torch.float64`` (the default) keeps neuron state,
        trajectories and adjoints in float64 (inputs and gradients stay
        float32); ``torch.float32`` keeps them in float32."""
        return BpttModel(self, trials, ms, readout, checkpoint_ms, smooth, device, state_dtype)


class BpttModel:
    """Device buffers of one differentiable network configuration (the
    native handle of nemo_b200_bptt_new)."""

    SMOOTH, FP64_STATE = 1, 2  # option bits of nemo_b200_bptt_new

    def __init__(self, net: DifferentiableNetwork, trials: int, ms: int, readout: int, checkpoint_ms: int,
                 smooth: bool, device: int | None, state_dtype: torch.dtype = torch.float64):
        if state_dtype not in (torch.float32, torch.float64):
            raise ValueError("state_dtype must be torch.float32 or torch.float64")
        self.net = net
        self.trials, self.ms, self.readout = trials, ms, readout
        self.state_dtype = state_dtype
        dev = torch.cuda.current_device() if device is None else device
        self.device = torch.device("cuda", dev)
        src = np.ascontiguousarray(net.source, np.uint32)
        tgt = np.ascontiguousarray(net.target, np.uint32)
        dly = np.ascontiguousarray(net.delay, np.uint32)
        options = (self.SMOOTH if smooth else 0) | (self.FP64_STATE if state_dtype == torch.float64 else 0)
        h = lib().nemo_b200_bptt_new(net.neurons, trials, ms, readout, checkpoint_ms, len(src), src, tgt, dly,
                                     options, dev)
        if not h:
            raise NemoError(lib().nemo_b200_last_status(), lib().nemo_strerror().decode())
        self._h = h
        # kept for __del__, which may run after this module's globals are gone
        self._delete = lib().nemo_b200_bptt_delete
        self.c, self.d = net.constants(self.device)

    def __del__(self):
        if getattr(self, "_h", None):
            self._delete(self._h)
            self._h = None

    def loss(self, W, a, b, noise, target):
        """Differentiable loss (a 0-d tensor); gradients flow to W, a, b."""
        return _IzhikevichBPTT.apply(W, a, b, noise, target, self)

    def _ptrs(self, *tensors):
        return [C.c_void_p(t.data_ptr()) for t in tensors]

    generation = 0  # forward passes run so far (the backward pass needs the latest one)

    def forward_raw(self, W, a, b, noise, target):
        self.generation += 1
        loss = torch.zeros(1, device=self.device, dtype=torch.float32)
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _check(lib().nemo_b200_bptt_forward(self._h, *self._ptrs(W, a, b, self.c, self.d, noise, target, loss), stream))
        return loss

    def readout_trains(self, W, a, b, noise) -> torch.Tensor:
        """Forward pass without a target; returns the filtered readout spike
        trains [ms, trials, readout] (a teacher's targets)."""
        target = torch.zeros((self.ms, self.trials, self.readout), device=self.device, dtype=torch.float32)
        with torch.no_grad():
            self.forward_raw(W, a, b, noise, target)
        out = torch.empty_like(target)
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _check(lib().nemo_b200_bptt_readout(self._h, C.c_void_p(out.data_ptr()), stream))
        return out

    def backward_raw(self, W, a, b, noise, target):
        dW = torch.empty_like(W)
        da = torch.empty_like(a)
        db = torch.empty_like(b)
        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _check(lib().nemo_b200_bptt_backward(self._h, *self._ptrs(W, a, b, self.c, self.d, noise, target, dW, da, db),
                                             stream))
        return dW, da, db


class _IzhikevichBPTT(torch.autograd.Function):
    """Forward and adjoint run by the native kernels; the backward pass
    differentiates the most recent forward pass of the same model."""

    @staticmethod
    def forward(ctx, W, a, b, noise, target, model: BpttModel):
        for t in (W, a, b, noise, target):
            if t.dtype != torch.float32 or not t.is_contiguous() or t.device != model.device:
                raise ValueError("float32 contiguous tensors on the model's device expected")
        ctx.model = model
        ctx.save_for_backward(W, a, b, noise, target)
        loss = model.forward_raw(W, a, b, noise, target)[0]
        ctx.generation = model.generation
        return loss

    @staticmethod
    def backward(ctx, grad):
        W, a, b, noise, target = ctx.saved_tensors
        if ctx.model.generation != ctx.generation:
            # another forward pass ran on this model since: redo ours
            ctx.model.forward_raw(W, a, b, noise, target)
        dW, da, db = ctx.model.backward_raw(W, a, b, noise, target)
        return dW * grad, da * grad, db * grad, None, None, None
