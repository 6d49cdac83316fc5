"""The oracle (the C restatement of the reference CPU backend) against the
reference's own known-answer tests and against the committed golden vectors.
CPU only."""
import os

import numpy as np
import pytest

import oracle as O
from tests import kat, nets

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("ncount,delay", [(1000, 1), (1024, 1), (2000, 1), (4000, 1), (2000, 20), (1000, 63)])
def test_ring(ncount, delay):
    kat.ring(O, ncount, delay)


def test_double_ring():
    kat.double_ring(O)


def test_firing_stimulus():
    kat.firing_stimulus(O)


def test_current_stimulus():
    kat.current_stimulus(O)


def test_invalid_current_stimulus():
    kat.invalid_current_stimulus(O)


def test_fixed_point_saturation():
    kat.fixed_point_saturation(O)


@pytest.mark.parametrize("n0,nstep", [(1, 1), (1000000, 1), (1, 4), (1000000, 4)])
def test_non_contiguous_indices(n0, nstep):
    kat.non_contiguous_indices(O, n0, nstep)


@pytest.mark.parametrize("iz_first", [True, False])
def test_neuron_type_mixture(iz_first):
    kat.neuron_type_mixture(O, iz_first)


@pytest.mark.parametrize("others", [False, True])
def test_poisson_rate(others):
    kat.poisson_rate(O, 10000, others)


@pytest.mark.parametrize("reward", [1.0, 0.8, 0.9])
def test_stdp_analytic(reward):
    kat.stdp_analytic(O, reward)


@pytest.mark.parametrize("ncount,iz", [(1, False), (1000, False), (1, True), (1000, True)])
def test_input_neurons(ncount, iz):
    kat.input_create(O, ncount, iz)
    kat.input_simple(O, ncount, iz, steps=300)


@pytest.mark.parametrize("reward", [1.0, 0.0])
def test_first_call_clamp(reward):
    kat.first_call_clamp(O, reward)


def test_zero_reward_clears_accumulators():
    kat.zero_reward_clears(O)


@pytest.mark.parametrize("stdp", [False, True])
def test_get_synapses(stdp):
    kat.get_synapses(O, stdp)


def test_write_only_synapses():
    kat.write_only_synapses(O)


def test_synapses_from_unconnected_neuron():
    kat.synapses_from_unconnected_neuron(O)


def test_high_firing():
    kat.high_firing(O, steps=100)


def test_vprobe():
    kat.vprobe(O)


def test_stdp_with_all_static():
    kat.stdp_with_all_static(O)


def test_set_neuron():
    kat.set_neuron_simulation(O)


def test_izhikevich_rs():
    kat.izhikevich_rs_no_parameters(O)
    stream, _ = kat.izhikevich_rs_network(O, steps=200)
    assert sum(len(f) for f in stream) > 500


def test_kuramoto():
    """src/test/Kuramoto.cpp against the analytic phases (the reference's
    0.001 % tolerance)"""
    kat.kuramoto_init(O)
    kat.kuramoto_uncoupled(O)
    kat.kuramoto_simple_coupled(O)
    for n, noise in [(2, False), (100, False), (100, True), (256, False)]:
        kat.kuramoto_n_to_1(O, n, noise)
    kat.kuramoto_with_stdp_fails(O)


def test_ring_delay_80_rejected():
    """The CPU backend rejects delays above 64 (src/nemo/cpu/Simulation.cpp:52-56)."""
    with pytest.raises(O.NemoError):
        O.Simulation(nets.create_ring(O, O.Network(), 2000, delay=80), O.Configuration())


def _load(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {name}; run tests/golden/make_golden.py")
    return np.load(path)


def test_golden_nrand():
    """The RNG restatement (src/nemo/RNG.cpp) against committed vectors: the
    seeds of local indices 0..63 and 1000..1063 and 64 nrand draws from each."""
    g = _load("rng.npz")
    assert np.array_equal(O.seed_states(0, 64), g["seeds0"])
    assert np.array_equal(O.seed_states(1000, 64), g["seeds1000"])
    st = g["seeds0"].copy()
    out = np.zeros((64, 64), np.float32)
    for i in range(64):
        s = st[i].copy()
        for k in range(64):
            out[i, k] = O.nrand(s)
    assert np.array_equal(out.view(np.uint32), g["nrand"].view(np.uint32))


def test_golden_random_1k():
    """The 1k x 100 random network, 1000 ms: fire stream and final state."""
    g = _load("random_1k.npz")
    sim = O.Simulation(O.example_random(1000, 100, 20, False), O.Configuration())
    counts, ids = sim.run(1000)
    assert np.array_equal(counts, g["counts"])
    assert np.array_equal(ids, g["ids"])
    assert np.array_equal(sim.type_state(0, 2, 1000).view(np.uint32), g["state"].view(np.uint32))


def test_golden_stdp_2k():
    """The 2000 x 200 random network with STDP, 500 ms with applyStdp every
    100 ms: fire stream and every weight."""
    g = _load("stdp_2k.npz")
    sim = O.Simulation(O.example_random(2000, 200, 20, True), nets.standard_stdp(O))
    counts, ids = sim.run(500, 100, 1.0)
    assert np.array_equal(counts, g["counts"])
    assert np.array_equal(ids, g["ids"])
    assert np.array_equal(sim.weights_fx(2000 * 200), g["weights"])
