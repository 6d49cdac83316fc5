"""The differentiable mode: the hand-written BPTT adjoint against PyTorch
autograd of the same unrolled dynamics in float64 (the FP64 oracle,
oracle/bptt_torch.py) and against finite differences of the smooth forward.

The relative error of a gradient vector is ||g - g64|| / ||g64||.  With
float64 state the adjoint must match the FP64 oracle to 1e-4.  With float32
state the gradient carries the rounding of a float32 evaluation, which the
spike upstroke amplifies (PyTorch's own float32 autograd of the same model
is off by about 1e-2 on these networks), so that mode must be no worse than
PyTorch float32 autograd on the same GPU."""
import numpy as np
import pytest
import torch

from nemosim_b200.bptt import DifferentiableNetwork
from oracle import bptt_torch as R

pytestmark = pytest.mark.gpu

TOL = 1e-4


def setup(neurons=256, fanout=24, ms=80, trials=4, readout=32, smooth=True, ckpt=20, seed=1,
          state_dtype=torch.float32):
    dev = torch.device("cuda", 0)
    net = DifferentiableNetwork.random(neurons, fanout, max_delay=10, seed=seed)
    teacher = DifferentiableNetwork.random(neurons, fanout, max_delay=10, seed=seed + 100)
    g = torch.Generator(device="cpu").manual_seed(seed)
    noise = (5.0 * torch.randn((ms, trials, neurons), generator=g)).to(dev)
    tmodel = teacher.model(trials, ms, readout, ckpt, smooth)
    Wt, at, bt = teacher.tensors(dev, requires_grad=False)
    target = tmodel.readout_trains(Wt, at, bt, noise)
    model = net.model(trials, ms, readout, ckpt, smooth, state_dtype=state_dtype)
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
    ref = ref.double()
    return float((x - ref).norm() / ref.norm().clamp_min(1e-300))


@pytest.mark.parametrize("smooth", [True, False])
def test_fp64_state_gradient_matches_fp64_autograd(smooth):
    dev, net, model, noise, target = setup(smooth=smooth, state_dtype=torch.float64)
    W, a, b = net.tensors(dev)
    loss = model.loss(W, a, b, noise, target)
    loss.backward()
    l64, gW, ga, gb = reference(net, dev, noise, target, 32, smooth)
    errs = [relerr(W.grad, gW), relerr(a.grad, ga), relerr(b.grad, gb)]
    print(f"smooth={smooth} fp64 state: loss {float(loss):.6g} vs {float(l64):.6g}; "
          f"rel. err. W {errs[0]:.2e} a {errs[1]:.2e} b {errs[2]:.2e}")
    assert abs(float(loss) - float(l64)) <= TOL * abs(float(l64))
    assert max(errs) <= TOL, errs


@pytest.mark.parametrize("smooth", [True, False])
def test_fp32_state_gradient_no_worse_than_fp32_autograd(smooth):
    dev, net, model, noise, target = setup(smooth=smooth)
    W, a, b = net.tensors(dev)
    loss = model.loss(W, a, b, noise, target)
    loss.backward()
    l64, gW, ga, gb = reference(net, dev, noise, target, 32, smooth)
    _, tW, ta, tb = reference(net, dev, noise, target, 32, smooth, dtype=torch.float32)
    ours = [relerr(W.grad, gW), relerr(a.grad, ga), relerr(b.grad, gb)]
    torch32 = [relerr(tW, gW), relerr(ta, ga), relerr(tb, gb)]
    print(f"smooth={smooth} fp32 state rel. err. {['%.2e' % e for e in ours]}, "
          f"torch fp32 autograd {['%.2e' % e for e in torch32]}")
    assert abs(float(loss) - float(l64)) <= TOL * abs(float(l64))
    for e, t in zip(ours, torch32):
        assert e <= max(TOL, 2.0 * t), (ours, torch32)


def test_gradient_matches_finite_differences():
    """Central differences of the smooth float64 forward along random
    directions agree with the adjoint's directional derivative (float64
    state).  a and b move every neuron at once, and the loss is smooth in
    them only on a scale of about 1e-6, hence the smaller step there."""
    dev, net, model, noise, target = setup(smooth=True, neurons=128, fanout=16, ms=60, state_dtype=torch.float64)
    W, a, b = net.tensors(dev)
    model.loss(W, a, b, noise, target).backward()
    c, d = net.constants(dev, dtype=torch.float64)
    st = R.Structure(net.source, net.target, net.delay, net.neurons, dev)
    W64, a64, b64 = (t.detach().double() for t in (W, a, b))
    n64, t64 = noise.double(), target.double()
    gen = torch.Generator(device="cpu").manual_seed(7)
    for name, base, grad, step in (("W", W64, W.grad, 1e-6), ("a", a64, a.grad, 1e-7), ("b", b64, b.grad, 1e-7)):
        direction = torch.randn(base.shape, generator=gen, dtype=torch.float64).to(dev)
        direction /= direction.norm()
        eps = step * max(1.0, float(base.abs().max()))
        args = {"W": W64, "a": a64, "b": b64}

        def f(x):
            kw = dict(args)
            kw[name] = x
            return float(R.loss(kw["W"], kw["a"], kw["b"], c, d, n64, t64, st, 32, True))
        fd = (f(base + eps * direction) - f(base - eps * direction)) / (2 * eps)
        ad = float((grad.double() * direction).sum())
        print(f"{name}: finite difference {fd:.8g}, adjoint {ad:.8g}")
        assert abs(fd - ad) <= 1e-3 * abs(fd) + 1e-12, (name, fd, ad)


@pytest.mark.parametrize("state_dtype", [torch.float32, torch.float64])
def test_checkpoint_interval_does_not_change_gradients(state_dtype):
    dev, net, model, noise, target = setup(smooth=True, ckpt=20, state_dtype=state_dtype)
    m2 = net.model(4, 80, 32, 7, True, state_dtype=state_dtype)
    W, a, b = net.tensors(dev)
    model.loss(W, a, b, noise, target).backward()
    W2, a2, b2 = net.tensors(dev)
    m2.loss(W2, a2, b2, noise, target).backward()
    assert torch.equal(W.grad, W2.grad) and torch.equal(a.grad, a2.grad) and torch.equal(b.grad, b2.grad)


def test_options_are_checked():
    from nemosim_b200 import NemoError, lib
    src = np.zeros(1, np.uint32)
    h = lib().nemo_b200_bptt_new(4, 1, 10, 1, 5, 1, src, src, np.ones(1, np.uint32), 4, 0)
    assert not h
    with pytest.raises(ValueError):
        DifferentiableNetwork.random(8, 2).model(1, 10, 1, state_dtype=torch.float16)
    assert NemoError is not None


def test_full_size_speed_vs_torch_autograd():
    """The differentiable configuration at full size (4096 neurons x 200
    synapses, 500 ms, 16 trials, 256 readouts, checkpoints every 50 ms): one
    gradient step of the adjoint, with float32 and with float64 state,
    against PyTorch float32 autograd of the same model on the same GPU."""
    import time
    dev, net, model, noise, target = setup(neurons=4096, fanout=200, ms=500, trials=16, readout=256,
                                           smooth=False, ckpt=50)
    times = {}
    for dtype in (torch.float32, torch.float64):
        m = net.model(16, 500, 256, 50, False, state_dtype=dtype)
        W, a, b = net.tensors(dev)
        for _ in range(2):
            W.grad = a.grad = b.grad = None
            m.loss(W, a, b, noise, target).backward()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            W.grad = a.grad = b.grad = None
            m.loss(W, a, b, noise, target).backward()
        torch.cuda.synchronize()
        times[dtype] = (time.perf_counter() - t0) / 3
        del m
    W32, a32, b32 = net.tensors(dev)
    c32, d32 = net.constants(dev)
    st = R.Structure(net.source, net.target, net.delay, net.neurons, dev)
    R.loss(W32, a32, b32, c32, d32, noise, target, st, 256, False).backward()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(2):
        W32.grad = a32.grad = b32.grad = None
        R.loss(W32, a32, b32, c32, d32, noise, target, st, 256, False).backward()
    torch.cuda.synchronize()
    theirs = (time.perf_counter() - t0) / 2
    ours32, ours64 = times[torch.float32], times[torch.float64]
    print(f"adjoint fp32 state {ours32 * 1e3:.1f} ms, fp64 state {ours64 * 1e3:.1f} ms, "
          f"torch autograd {theirs * 1e3:.1f} ms, speedup {theirs / ours32:.1f}x / {theirs / ours64:.1f}x")
    assert theirs / ours32 >= 10.0
    assert theirs / ours64 >= 10.0


def test_full_size_accuracy_vs_fp64_autograd():
    """The gradient error at full size (4096 x 200, 500 ms, 16 trials, 256
    readouts, hard threshold): the adjoint with float64 state within TOL of
    float64 autograd, and with float32 state no worse than twice PyTorch's
    own float32 autograd of the same model (both against float64)."""
    dev, net, _, noise, target = setup(neurons=4096, fanout=200, ms=500, trials=16, readout=256,
                                       smooth=False, ckpt=50)
    l64, gW, ga, gb = reference(net, dev, noise, target, 256, False)
    _, tW, ta, tb = reference(net, dev, noise, target, 256, False, dtype=torch.float32)
    torch32 = [relerr(tW, gW), relerr(ta, ga), relerr(tb, gb)]
    del tW, ta, tb
    errs = {}
    for dtype in (torch.float64, torch.float32):
        m = net.model(16, 500, 256, 50, False, state_dtype=dtype)
        W, a, b = net.tensors(dev)
        loss = m.loss(W, a, b, noise, target)
        loss.backward()
        errs[dtype] = (abs(float(loss) - float(l64)) / abs(float(l64)),
                       [relerr(W.grad, gW), relerr(a.grad, ga), relerr(b.grad, gb)])
        del m
    for dtype, (lerr, e) in errs.items():
        print(f"full size, {dtype} state: loss rel. err. {lerr:.2e}; gradient rel. err. W {e[0]:.2e} "
              f"a {e[1]:.2e} b {e[2]:.2e}")
    print(f"full size, torch float32 autograd: W {torch32[0]:.2e} a {torch32[1]:.2e} b {torch32[2]:.2e}")
    lerr64, e64 = errs[torch.float64]
    assert lerr64 <= TOL and max(e64) <= TOL, e64
    lerr32, e32 = errs[torch.float32]
    assert lerr32 <= TOL
    for e, t in zip(e32, torch32):
        assert e <= max(TOL, 2.0 * t), (e32, torch32)
