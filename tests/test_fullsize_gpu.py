"""Bit-exact parity with the oracle at the full sizes of the benchmark
configurations.

- The 100,000-neuron x 1000-synapse random network (src/examples/random.cpp)
  with STDP (20 + 20 ms window, A+ = 0.1, A- = -0.12, weights [0, 10],
  applyStdp(1.0) every 100 ms), maximum delay 44, for its first 1000 ms:
  the fire stream, the fp32 state of every neuron and all 100M Q11.20
  weights.
- The mixed-plugin network: 50,000 IF_curr_exp + 50,000 Izhikevich + 10,000
  PoissonSource (5 Hz), Pareto(1.5) out-degree with mean 500 capped at
  10,000, lognormal(-1, 1) weights with 20% of the signs flipped, delays
  1-32 ms, 2000 ms: the fire stream and the fp32 state of both stateful
  types.

Each side runs alone and is deleted before the other is built, so that the
host holds one copy of the network at a time.

- The 256-network batch of the batched configuration, 1000 ms: every
  network's fire stream in the batch equals its own single-network run
  (which the parity tests above pin to the oracle's arithmetic).
"""
import gc

import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

pytestmark = pytest.mark.gpu

f32 = np.float32


def same_bits(a, b) -> bool:
    a = np.asarray(a, f32)
    b = np.asarray(b, f32)
    if a.shape != b.shape:
        return False
    nan = np.isnan(a) & np.isnan(b)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | nan))


def first_difference(a, b) -> str:
    if a.shape != b.shape:
        return f"shapes differ: {a.shape} vs {b.shape}"
    k = int(np.argmax(a != b))
    return f"first difference at {k}: {a[k]} vs {b[k]}"


def test_c2_100k_x_1000_stdp_first_1000_ms():
    N, F, D, MS, PERIOD = 100_000, 1000, 44, 1000, 100

    def run(mod):
        sim = mod.Simulation(mod.example_random(N, F, D, True), nets.standard_stdp(mod))
        w0 = sim.weights_fx(N * F)
        if mod is nb:
            counts, _, ids = sim.run(MS, PERIOD, 1.0, max_ids=MS * N // 20)
        else:
            counts, ids = sim.run(MS, PERIOD, 1.0, max_ids=MS * N // 20)
        out = (counts.copy(), ids, sim.type_state(0, 2, N), sim.weights_fx(N * F), w0)
        del sim
        gc.collect()
        return out

    cp, ip, sp, wp, w0p = run(nb)
    co, io, so, wo, w0o = run(O)
    assert np.array_equal(w0p, w0o), "initial weights: " + first_difference(w0p, w0o)
    assert cp.sum() > 100_000, "the network hardly fired"
    assert np.array_equal(cp, co), "fired counts: " + first_difference(cp, co)
    assert np.array_equal(ip, io), "fired ids: " + first_difference(ip, io)
    assert same_bits(sp, so), "neuron state differs"
    assert len(wp) == len(wo) == N * F
    assert np.array_equal(wp, wo), "weights: " + first_difference(wp, wo)
    # the ten applyStdp calls changed weights
    changed = int(np.count_nonzero(wp != w0p))
    assert changed > 10_000, changed


def test_c3_mixed_plugins_full_size_2000_ms():
    MS = 2000
    sizes = dict(n_if=50_000, n_iz=50_000, n_poisson=10_000, seed=7, mean_out=500, cap=10_000, dmax=32)

    def run(mod):
        net, types, ids = nets.mixed_network(mod, **sizes)
        sim = mod.Simulation(net, mod.Configuration())
        del net
        gc.collect()
        cap = MS * 110_000 // 2
        if mod is nb:
            counts, _, fired = sim.run(MS, max_ids=cap)
        else:
            counts, fired = sim.run(MS, max_ids=cap)
        states = [sim.type_state(types[0], 4, len(ids[0])), sim.type_state(types[1], 2, len(ids[1]))]
        out = (counts.copy(), fired, states)
        del sim
        gc.collect()
        return out

    cp, ip, sp = run(nb)
    co, io, so = run(O)
    assert cp.sum() > 1_000_000, "the network hardly fired"
    assert np.array_equal(cp, co), "fired counts: " + first_difference(cp, co)
    assert np.array_equal(ip, io), "fired ids: " + first_difference(ip, io)
    assert same_bits(sp[0], so[0]), "IF_curr_exp state differs"
    assert same_bits(sp[1], so[1]), "Izhikevich state differs"


def test_c4_256_network_batch_matches_individual_runs():
    """The batched configuration at full size: 256 networks of 1,000-32,000
    Izhikevich neurons, fan-out 100-1000, delays 1-20, input-noise sigma
    U(2, 8) and their own generator seeds (the benchmark's networks), 1000
    ms.  Every network's fire stream in the batch equals its own
    single-network run, bit for bit, and the batch is built on the device."""
    rng = np.random.default_rng(0)
    specs = [dict(n=int(rng.integers(1000, 32001)), f=int(rng.integers(100, 1001)), seed=1000 + 17 * k,
                  sigma=float(rng.uniform(2.0, 8.0))) for k in range(256)]
    MS = 1000

    def make(sp):
        return nb.example_random(sp["n"], sp["f"], 20, False, seed=sp["seed"], sigma_exc=sp["sigma"],
                                 sigma_inh=sp["sigma"])

    conf = nb.Configuration()
    singles, networks = [], []
    for sp in specs:
        net = make(sp)
        sim = nb.Simulation(net, conf)
        c, _, ids = sim.run(MS, max_ids=sp["n"] * MS // 10)
        singles.append((c, ids))
        del sim
        networks.append(net)
    batch = nb.Batch(networks, conf)
    del networks
    gc.collect()
    assert batch.connectivity_digest()[1]
    neurons = sum(sp["n"] for sp in specs)
    counts, _, ids = batch.run(MS, max_ids=neurons * MS // 20)
    streams = batch.streams(counts, ids)
    bad = [k for k, ((c1, i1), (c2, i2)) in enumerate(zip(streams, singles))
           if not (np.array_equal(c1, c2) and np.array_equal(i1, i2))]
    assert not bad, bad[:10]
    assert sum(int(c.sum()) for c, _ in singles) > 0
