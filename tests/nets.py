"""Network builders shared by the tests.  Each takes a module (the product
package ``nemosim_b200`` or the oracle package) and builds the same network
through that module's Network API, so both consume identical inputs.  The
builders restate the reference's test networks (src/test/utils.cpp,
src/test/stdp.cpp, src/test/test.cpp)."""
from __future__ import annotations

import numpy as np

f32 = np.float32


def ring_neuron_args():
    """createRing's neuron (src/test/utils.cpp:136-141)."""
    v = f32(-65.0)
    b = f32(0.2)
    r = f32(0.5)
    r2 = f32(r * r)
    return (f32(0.02), b, f32(v + f32(15.0) * r2), f32(f32(8.0) - f32(6.0) * r2), f32(0.0), f32(b * v), v)


def create_ring(mod, net, ncount, n0=0, plastic=False, nstep=1, delay=1):
    """createRing (src/test/utils.cpp:132-145): neuron i -> i+1 with weight 1000."""
    iz = net.add_neuron_type("Izhikevich")
    a, b, c, d, sigma, u, v = ring_neuron_args()
    idx = np.array([n0 + (i % ncount) * nstep for i in range(ncount)], np.uint32)
    tgt = np.array([n0 + ((i + 1) % ncount) * nstep for i in range(ncount)], np.uint32)
    net.add_neuron(iz, idx, a, b, c, d, sigma, u, v)
    net.add_synapse(idx, tgt, np.full(ncount, delay, np.uint32), np.full(ncount, 1000.0, np.float32),
                    np.full(ncount, bool(plastic), np.uint8))
    return net


def exc_neuron_args(sigma=0.0):
    """addExcitatoryNeuron of src/test/utils.cpp:106-113."""
    r = f32(0.5)
    b = f32(f32(0.25) - f32(0.05) * r)
    v = f32(-65.0)
    return (f32(f32(0.02) + f32(0.08) * r), b, v, f32(2.0), f32(sigma), f32(b * v), v)


def stdp_test_configuration(mod):
    """configuration() of src/test/stdp.cpp:76-97."""
    conf = mod.Configuration()
    pre = np.array([f32(1.0) * np.exp(f32(-dt) / f32(20.0), dtype=f32) for dt in range(20)], f32)
    post = np.array([f32(-0.8) * np.exp(f32(-dt) / f32(20.0), dtype=f32) for dt in range(20)], f32)
    conf.set_stdp_function(pre, post, -0.5, 2 * 5.0)
    return conf


def standard_stdp(mod, a_plus=0.1, a_minus=-0.12, tau=20.0, n=20, wmax=10.0):
    """The benchmark STDP window (exponential, dt = 1..n) with weights in
    [0, wmax] for excitatory synapses and [-wmax, 0] for inhibitory ones."""
    conf = mod.Configuration()
    dt = np.arange(1, n + 1, dtype=f32)
    pre = (f32(a_plus) * np.exp(-dt / f32(tau))).astype(f32)
    post = (f32(a_minus) * np.exp(-dt / f32(tau))).astype(f32)
    conf.set_stdp_function(pre, post, -wmax, wmax)
    return conf


def mixed_network(mod, n_if=500, n_iz=500, n_poisson=100, seed=7, mean_out=50, cap=1000, dmax=32):
    """A scaled-down mixed-plugin network with Pareto out-degree, lognormal
    weights (20% sign-flipped) and uniform delays: 50k IF_curr_exp + 50k
    Izhikevich + 10k Poisson at 5 Hz in its full-size form."""
    rng = np.random.default_rng(seed)
    net = mod.Network()
    tif = net.add_neuron_type("IF_curr_exp")
    tiz = net.add_neuron_type("Izhikevich")
    tps = net.add_neuron_type("PoissonSource")
    n = n_if + n_iz + n_poisson
    ids = rng.permutation(n).astype(np.uint32)  # non-contiguous, interleaved ids
    if_ids, iz_ids, ps_ids = ids[:n_if], ids[n_if:n_if + n_iz], ids[n_if + n_iz:]
    # IF_curr_exp: v_rest, v_reset, c_m, tau_m, tau_refrac, tau_synE, tau_synI, v_thresh, i_offset | v, Ie, Ii, lastfired
    net.add_neuron(tif, if_ids, -65.0, -65.0, 1.0, 20.0, 2.0, 5.0, 5.0, -50.0, 0.0, -65.0, 0.0, 0.0, 1000.0)
    r1 = rng.random(n_iz).astype(f32)
    r2 = rng.random(n_iz).astype(f32)
    exc = rng.random(n_iz) < 0.8
    a = np.where(exc, f32(0.02), f32(0.02) + f32(0.08) * r1).astype(f32)
    b = np.where(exc, f32(0.2), f32(0.25) - f32(0.05) * r2).astype(f32)
    c = np.where(exc, f32(-65.0) + f32(15.0) * r1 * r1, f32(-65.0)).astype(f32)
    d = np.where(exc, f32(8.0) - f32(6.0) * r2 * r2, f32(2.0)).astype(f32)
    sigma = np.where(exc, f32(5.0), f32(2.0)).astype(f32)
    net.add_neuron(tiz, iz_ids, a, b, c, d, sigma, (b * f32(-65.0)).astype(f32), f32(-65.0))
    net.add_neuron(tps, ps_ids, f32(0.005))
    # Pareto(alpha=1.5) out-degree with the given mean, capped
    alpha = 1.5
    xm = mean_out * (alpha - 1) / alpha
    deg = np.minimum((xm / rng.random(n) ** (1 / alpha)).astype(np.int64), cap)
    src = np.repeat(ids, deg).astype(np.uint32)
    tgt = ids[rng.integers(0, n, len(src))].astype(np.uint32)
    w = rng.lognormal(-1.0, 1.0, len(src)).astype(f32)
    w = np.where(rng.random(len(src)) < 0.2, -w, w).astype(f32)
    dly = rng.integers(1, dmax + 1, len(src)).astype(np.uint32)
    net.add_synapse(src, tgt, dly, w, np.zeros(len(src), np.uint8))
    return net, (tif, tiz, tps), (if_ids, iz_ids, ps_ids)
