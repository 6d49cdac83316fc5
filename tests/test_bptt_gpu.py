"""The differentiable mode: the hand-written BPTT adjoint against PyTorch
autograd of the same unrolled dynamics in float64 (the FP64 oracle,
oracle/bptt_torch.py) and against finite differences of the smooth forward.
The tolerance is a relative error of 1e-4 on the gradient vectors
(||g - g64|| / ||g64||)."""
import numpy as np
import pytest
import torch

from nemosim_b200.bptt import DifferentiableNetwork
from oracle import bptt_torch as R

pytestmark = pytest.mark.gpu

TOL = 1e-4


def setup(neurons=256, fanout=24, ms=80, trials=4, readout=32, smooth=True, ckpt=20, seed=1):
    dev = torch.device("cuda", 0)
    net = DifferentiableNetwork.random(neurons, fanout, max_delay=10, seed=seed)
    teacher = DifferentiableNetwork.random(neurons, fanout, max_delay=10, seed=seed + 100)
    g = torch.Generator(device="cpu").manual_seed(seed)
    noise = (5.0 * torch.randn((ms, trials, neurons), generator=g)).to(dev)
    tmodel = teacher.model(trials, ms, readout, ckpt, smooth)
    Wt, at, bt = teacher.tensors(dev, requires_grad=False)
    target = tmodel.readout(Wt, at, bt, noise)
    model = net.model(trials, ms, readout, ckpt, smooth)
    return dev, net, model, noise, target


def reference(net, dev, noise, target, readout, smooth, dtype=torch.float64):
    W, a, b = net.tensors(dev, dtype=dtype)
    c, d = net.constants(dev, dtype=dtype)
    st = R.Structure(net.source, net.target, net.delay, net.neurons, dev)
    loss = R.loss(W, a, b, c, d, noise.to(dtype), target.to(dtype), st, readout, smooth)
    loss.backward()
    return loss.detach(), W.grad, a.grad, b.grad


def relerr(x, ref):
    x = x.double()
    return float((x - ref).norm() / ref.norm().clamp_min(1e-300))


@pytest.mark.parametrize("smooth", [True, False])
def test_gradient_matches_fp64_autograd(smooth):
    dev, net, model, noise, target = setup(smooth=smooth)
    W, a, b = net.tensors(dev)
    loss = model.loss(W, a, b, noise, target)
    loss.backward()
    l64, gW, ga, gb = reference(net, dev, noise, target, 32, smooth)
    assert abs(float(loss) - float(l64)) <= TOL * abs(float(l64))
    assert relerr(W.grad, gW) <= TOL, relerr(W.grad, gW)
    assert relerr(a.grad, ga) <= TOL, relerr(a.grad, ga)
    assert relerr(b.grad, gb) <= TOL, relerr(b.grad, gb)


def test_gradient_matches_finite_differences():
    """Central differences of the smooth float64 forward along random
    directions agree with the adjoint's directional derivative."""
    dev, net, model, noise, target = setup(smooth=True, neurons=128, fanout=16, ms=60)
    W, a, b = net.tensors(dev)
    model.loss(W, a, b, noise, target).backward()
    c, d = net.constants(dev, dtype=torch.float64)
    st = R.Structure(net.source, net.target, net.delay, net.neurons, dev)
    W64, a64, b64 = (t.detach().double() for t in (W, a, b))
    n64, t64 = noise.double(), target.double()
    gen = torch.Generator(device="cpu").manual_seed(7)
    for name, base, grad in (("W", W64, W.grad), ("a", a64, a.grad), ("b", b64, b.grad)):
        direction = torch.randn(base.shape, generator=gen, dtype=torch.float64).to(dev)
        direction /= direction.norm()
        eps = 1e-6 * max(1.0, float(base.abs().max()))
        args = {"W": W64, "a": a64, "b": b64}

        def f(x):
            kw = dict(args)
            kw[name] = x
            return float(R.loss(kw["W"], kw["a"], kw["b"], c, d, n64, t64, st, 32, True))
        fd = (f(base + eps * direction) - f(base - eps * direction)) / (2 * eps)
        ad = float((grad.double() * direction).sum())
        assert abs(fd - ad) <= 1e-3 * abs(fd) + 1e-12, (name, fd, ad)


def test_checkpoint_interval_does_not_change_gradients():
    dev, net, model, noise, target = setup(smooth=True, ckpt=20)
    m2 = net.model(4, 80, 32, 7, True)
    W, a, b = net.tensors(dev)
    model.loss(W, a, b, noise, target).backward()
    W2, a2, b2 = net.tensors(dev)
    m2.loss(W2, a2, b2, noise, target).backward()
    assert torch.equal(W.grad, W2.grad) and torch.equal(a.grad, a2.grad) and torch.equal(b.grad, b2.grad)


def test_full_size_speed_vs_torch_autograd():
    """The differentiable configuration at full size (4096 neurons x 200
    synapses, 500 ms, 16 trials, 256 readouts, checkpoints every 50 ms): one
    gradient step of the adjoint against PyTorch autograd (float32, same GPU)."""
    import time
    dev, net, model, noise, target = setup(neurons=4096, fanout=200, ms=500, trials=16, readout=256,
                                           smooth=False, ckpt=50)
    W, a, b = net.tensors(dev)
    for _ in range(2):
        W.grad = a.grad = b.grad = None
        model.loss(W, a, b, noise, target).backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        W.grad = a.grad = b.grad = None
        model.loss(W, a, b, noise, target).backward()
    torch.cuda.synchronize()
    ours = (time.perf_counter() - t0) / 3
    W32, a32, b32 = net.tensors(dev)
    c32, d32 = net.constants(dev)
    st = R.Structure(net.source, net.target, net.delay, net.neurons, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    R.loss(W32, a32, b32, c32, d32, noise, target, st, 256, False).backward()
    torch.cuda.synchronize()
    theirs = time.perf_counter() - t0
    print(f"adjoint {ours * 1e3:.1f} ms, torch autograd {theirs * 1e3:.1f} ms, speedup {theirs / ours:.1f}x")
    assert theirs / ours >= 10.0
