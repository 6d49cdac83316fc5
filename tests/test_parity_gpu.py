"""Parity of the B200 backend (through its C ABI) with the CPU oracle and with
the reference's own known-answer tests (src/test/test.cpp, src/test/stdp.cpp,
src/test/PoissonSource.cpp).  The bar is bit-exactness: identical fire
streams (cycle, neuron id), identical fp32 neuron state (NaN compared as NaN)
and identical fixed-point weights."""
import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import kat, nets

pytestmark = pytest.mark.gpu

f32 = np.float32


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    a = np.asarray(a, f32)
    b = np.asarray(b, f32)
    if a.shape != b.shape:
        return False
    nan = np.isnan(a) & np.isnan(b)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | nan))


def run_both(mod_nets, steps, stdp_period=0, reward=1.0):
    """Run product and oracle simulations and return their streams."""
    (sim_p, sim_o) = mod_nets
    cp, _, ip = sim_p.run(steps, stdp_period, reward, max_ids=steps * 20000)
    co, io = sim_o.run(steps, stdp_period, reward, max_ids=steps * 20000)
    return (cp, ip), (co, io)


def assert_streams_equal(p, o):
    cp, ip = p
    co, io = o
    if not np.array_equal(cp, co):
        t = int(np.argmax(cp != co))
        raise AssertionError(f"fired counts differ first at cycle {t}: {cp[t]} vs {co[t]}")
    if not np.array_equal(ip, io):
        k = int(np.argmax(ip != io))
        raise AssertionError(f"fired ids differ first at position {k}: {ip[k]} vs {io[k]}")


# ---------------------------------------------------------------------------
# known-answer tests of the reference (src/test/test.cpp), on the device

@pytest.mark.parametrize("ncount,delay", [(1000, 1), (1024, 1), (2000, 1), (4000, 1), (2000, 20), (1000, 63)])
def test_ring(ncount, delay):
    kat.ring(nb, ncount, delay)


def test_double_ring():
    kat.double_ring(nb)


def test_firing_stimulus():
    kat.firing_stimulus(nb)


def test_current_stimulus():
    kat.current_stimulus(nb)


def test_invalid_current_stimulus():
    kat.invalid_current_stimulus(nb)


def test_fixed_point_saturation():
    """... and bit-exact against the oracle"""
    assert same_bits(kat.fixed_point_saturation(nb), kat.fixed_point_saturation(O))


@pytest.mark.parametrize("n0,nstep", [(1, 1), (1000000, 1), (1, 4), (1000000, 4)])
def test_non_contiguous_indices(n0, nstep):
    kat.non_contiguous_indices(nb, n0, nstep)


@pytest.mark.parametrize("iz_first", [True, False])
def test_neuron_type_mixture(iz_first):
    """... and the Poisson firing is bit-exact against the oracle"""
    assert kat.neuron_type_mixture(nb, iz_first) == kat.neuron_type_mixture(O, iz_first)


@pytest.mark.parametrize("others", [False, True])
def test_poisson_rate(others):
    assert kat.poisson_rate(nb, 10000, others) == kat.poisson_rate(O, 10000, others)


@pytest.mark.parametrize("ncount,iz", [(1, False), (1000, False), (1, True), (1000, True)])
def test_input_neurons(ncount, iz):
    """The Input type (src/test/Input.cpp:41-79): it fires exactly when
    stimulated; the fire stream equals the oracle's"""
    kat.input_create(nb, ncount, iz)
    assert kat.input_simple(nb, ncount, iz) == kat.input_simple(O, ncount, iz)


@pytest.mark.parametrize("reward", [1.0, 0.0])
def test_first_call_clamp(reward):
    """The first applyStdp clamps weights that start outside the limits,
    with any reward (zero included)"""
    assert kat.first_call_clamp(nb, reward) == kat.first_call_clamp(O, reward)


def test_zero_reward_clears_accumulators():
    """applyStdp(0) clears the accumulators, keeps the weights, and later
    calls continue as on the oracle"""
    assert kat.zero_reward_clears(nb) == kat.zero_reward_clears(O)


@pytest.mark.parametrize("stdp", [False, True])
def test_get_synapses(stdp):
    """testGetSynapses (src/test/test.cpp:562-603): the simulation's synapse
    ids, targets, delays, weights and plasticity, equal to the network's and
    to the oracle's"""
    assert kat.get_synapses(nb, stdp) == kat.get_synapses(O, stdp)


def test_get_synapses_after_stdp():
    """Weights read back one by one after applyStdp equal the oracle's and
    the bulk read-back"""
    sims = [m.Simulation(m.example_random(1000, 100, 20, True), nets.standard_stdp(m)) for m in (nb, O)]
    for s in sims:
        s.run(300, 100, 1.0)
    for src in range(0, 1000, 37):
        ids = sims[0].get_synapses_from(src)
        assert list(ids) == list(sims[1].get_synapses_from(src))
        assert [sims[0].get_synapse_weight(i) for i in ids] == [sims[1].get_synapse_weight(i) for i in ids]
    assert np.array_equal(sims[0].weights_fx(100000), sims[1].weights_fx(100000))


def test_write_only_synapses():
    kat.write_only_synapses(nb)


def test_synapses_from_unconnected_neuron():
    kat.synapses_from_unconnected_neuron(nb)


def test_high_firing():
    """testHighFiring (src/test/test.cpp:697-736): every neuron fires every
    step, all delivery groups pending; state bit-exact with the oracle"""
    assert same_bits(kat.high_firing(nb), kat.high_firing(O))


def test_vprobe():
    kat.vprobe(nb)


def test_stdp_with_all_static():
    """testStdpWithAllStatic (src/test/test.cpp:666-680), fire stream equal
    to the oracle's"""
    assert kat.stdp_with_all_static(nb) == kat.stdp_with_all_static(O)


def test_set_neuron():
    """testSetNeuron (src/test/test.cpp:769-963) during simulation; every
    membrane potential it observes equal to the oracle's"""
    assert kat.set_neuron_simulation(nb) == kat.set_neuron_simulation(O)


def test_izhikevich_rs_no_parameters():
    """testNoParamNeuronType (src/test/test.cpp:980-1000), state bit-exact
    with the oracle's restatement of the reference's IzhikevichRS plugin"""
    assert same_bits(kat.izhikevich_rs_no_parameters(nb), kat.izhikevich_rs_no_parameters(O))


@pytest.mark.parametrize("resident", [True, False])
def test_izhikevich_rs_network(resident):
    """A connected, stimulated IzhikevichRS network, stepped through the
    resident loop or two launches per step: fire stream and state bit-exact
    with the oracle"""
    p = kat.izhikevich_rs_network(nb, resident=resident)
    o = kat.izhikevich_rs_network(O)
    assert sum(len(f) for f in p[0]) > 2000
    assert p[0] == o[0]
    assert same_bits(p[1], o[1])


def test_kuramoto_known_answers():
    """src/test/Kuramoto.cpp on the device, against the analytic phases with
    the reference's 0.001 % tolerance; STDP with a type that reads its
    sources is refused with NEMO_API_UNSUPPORTED"""
    kat.kuramoto_init(nb)
    kat.kuramoto_uncoupled(nb)
    kat.kuramoto_simple_coupled(nb)
    for n, noise in [(2, False), (100, False), (100, True), (256, False)]:
        kat.kuramoto_n_to_1(nb, n, noise)
    assert kat.kuramoto_with_stdp_fails(nb) == 5


@pytest.mark.parametrize("persistent", [True, False])
def test_kuramoto_matches_oracle(persistent):
    """A 2048-oscillator network with delayed couplings, 300 steps: the
    phases agree with the oracle's to 1e-4 radian.  Not bit for bit: the
    device's sinf is CUDA's, the oracle's the host libm's."""
    class Persistent:
        def __init__(self, on):
            self.on = on

        def __getattr__(self, name):
            return getattr(nb, name)

        def Simulation(self, net, conf):
            sim = nb.Simulation(net, conf)
            sim.set_persistent(self.on)
            return sim

    mod = Persistent(persistent)
    p = kat.kuramoto_random(mod, steps=300)
    o = kat.kuramoto_random(O, steps=300)
    d = np.abs(((p.astype(np.float64) - o + np.pi) % (2 * np.pi)) - np.pi)
    assert d.max() < 1e-4, d.max()


def test_kuramoto_source_and_delay_checks():
    """A Kuramoto oscillator reads its sources' phases from its own type's
    32-step history: other sources, or delays above 31, are refused"""
    net, k = kat.oscillator_network(nb)
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(k, 0, 0.1, 0.0)
    net.add_neuron(iz, 1, *nets.exc_neuron_args())
    net.add_synapse(1, 0, 1, 1.0, False)
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, nb.Configuration())
    assert e.value.code == 6
    net, k = kat.oscillator_network(nb)
    net.add_neuron(k, 0, 0.1, 0.0)
    net.add_neuron(k, 1, 0.1, 1.0)
    net.add_synapse(1, 0, 32, 1.0, False)
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, nb.Configuration())
    assert e.value.code == 6


# ---------------------------------------------------------------------------
# bit-exact parity with the oracle on noisy networks


def test_random_1k_bitexact():
    """The 1000-neuron x 100-synapse random network (src/examples/random.cpp,
    delays 1-20, STDP off), 1000 ms: fire stream and final state."""
    sims = (nb.Simulation(nb.example_random(1000, 100, 20, False), nb.Configuration()),
            O.Simulation(O.example_random(1000, 100, 20, False), O.Configuration()))
    p, o = run_both(sims, 1000)
    assert p[0].sum() > 1000
    assert_streams_equal(p, o)
    assert same_bits(sims[0].type_state(0, 2, 1000), sims[1].type_state(0, 2, 1000))


def test_step_matches_run():
    """nemo_step (one host round trip per ms) and the device-resident run give
    the same stream."""
    a = nb.Simulation(nb.example_random(1000, 100, 20, False), nb.Configuration())
    b = nb.Simulation(nb.example_random(1000, 100, 20, False), nb.Configuration())
    counts, _, ids = a.run(300)
    stream = []
    for _ in range(300):
        stream.extend(b.step())
    assert np.array_equal(ids, np.array(stream, np.uint32))
    assert counts.sum() == len(stream)


@pytest.mark.parametrize("persistent", [True, False])
def test_stdp_bitexact(persistent):
    """A 2000 x 200 random network with STDP (delays 1-20, window 20+20,
    applyStdp(1.0) every 100 ms): fire stream, state and every weight, with
    the persistent step loop and with the two-launch step."""
    sims = (nb.Simulation(nb.example_random(2000, 200, 20, True), nets.standard_stdp(nb)),
            O.Simulation(O.example_random(2000, 200, 20, True), nets.standard_stdp(O)))
    sims[0].set_persistent(persistent)
    p, o = run_both(sims, 1000, stdp_period=100)
    assert_streams_equal(p, o)
    nsyn = 2000 * 200
    wp, wo = sims[0].weights_fx(nsyn), sims[1].weights_fx(nsyn)
    assert not np.array_equal(wp, O.example_random(2000, 200, 20, True).synapses()[3])  # weights did change
    assert np.array_equal(wp, wo)
    assert same_bits(sims[0].type_state(0, 2, 2000), sims[1].type_state(0, 2, 2000))


@pytest.mark.parametrize("persistent", [True, False])
def test_stdp_inflight_compensation(persistent):
    """applyStdp between a spike's emission and its arrival: the arriving
    weight is the updated one (long delays, frequent applyStdp)."""
    sims = (nb.Simulation(nb.example_random(1500, 150, 40, True), nets.standard_stdp(nb, n=20)),
            O.Simulation(O.example_random(1500, 150, 40, True), nets.standard_stdp(O, n=20)))
    sims[0].set_persistent(persistent)
    p, o = run_both(sims, 600, stdp_period=7, reward=0.8)
    assert_streams_equal(p, o)
    assert np.array_equal(sims[0].weights_fx(1500 * 150), sims[1].weights_fx(1500 * 150))


def test_mixed_plugins_bitexact():
    """IF_curr_exp + Izhikevich + Poisson with Pareto out-degree and mixed-sign
    lognormal weights (the mixed-plugin configuration, scaled down)."""
    (np_, tp, idp) = nets.mixed_network(nb)
    (no_, to, ido) = nets.mixed_network(O)
    sims = (nb.Simulation(np_, nb.Configuration()), O.Simulation(no_, O.Configuration()))
    p, o = run_both(sims, 1000)
    assert p[0].sum() > 0
    assert_streams_equal(p, o)
    for t, ns, n in [(tp[0], 4, len(idp[0])), (tp[1], 2, len(idp[1]))]:
        assert same_bits(sims[0].type_state(t, ns, n), sims[1].type_state(t, ns, n))


@pytest.mark.parametrize("persistent", [True, False])
@pytest.mark.parametrize("shape", [(32, 32), (64, 64), (96, 128), (256, 128), (1024, 256), (2048, 1024)])
def test_launch_shape_does_not_change_results(shape, persistent):
    """Any partition size / block size gives the same bit-exact results, in
    either step-loop mode (the reference simulation uses the default)."""
    ref = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    sim = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    sim.set_persistent(persistent)
    sim.set_launch(*shape)
    assert sim.launch()[0] == shape[0]
    a = ref.run(300, 100, 1.0)
    b = sim.run(300, 100, 1.0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    assert np.array_equal(ref.weights_fx(450000), sim.weights_fx(450000))


def test_graph_replay_matches_single_launches():
    """The two-launch step loop replays 100-step CUDA graphs from a device
    cycle counter; the results equal single launches, across applyStdp calls
    and remainders."""
    a = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    a.set_persistent(False)
    b.set_persistent(False)
    b.set_graphs(False)
    for steps, period in [(537, 100), (250, 0), (333, 70)]:
        ra = a.run(steps, period, 1.0)
        rb = b.run(steps, period, 1.0)
        assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[2], rb[2])
    a.set_launch(64, 64)  # the graph is rebuilt for the new shape
    b.set_launch(64, 64)
    ra = a.run(300, 100, 1.0)
    rb = b.run(300, 100, 1.0)
    assert np.array_equal(ra[2], rb[2])
    assert np.array_equal(a.weights_fx(450000), b.weights_fx(450000))


def test_persistent_loop_matches_two_launch_step():
    """The persistent step loop (one cooperative launch per segment between
    applyStdp calls) equals the two-launch step, across applyStdp calls,
    remainders, single-step segments and interleaved nemo_step calls."""
    a = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b.set_persistent(False)
    for steps, period in [(537, 100), (250, 0), (333, 70), (5, 1), (101, 2)]:
        ra = a.run(steps, period, 1.0)
        rb = b.run(steps, period, 1.0)
        assert np.array_equal(ra[0], rb[0]) and np.array_equal(ra[2], rb[2])
        assert list(a.step()) == list(b.step())
    assert np.array_equal(a.weights_fx(450000), b.weights_fx(450000))
    assert same_bits(a.type_state(0, 2, 3000), b.type_state(0, 2, 3000))


def test_phase_trace_advances_like_run():
    """The phase trace runs the persistent loop like run() does: the
    simulation continues identically afterwards, and every CTA's marks are
    in order within each step."""
    a = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    a.run(100, 100, 1.0)
    b.run(100, 100, 1.0)
    tr = a.trace_phases(100)
    b.run(100)  # the traced launch is a run's launch without applyStdp
    assert tr.shape[0] == 100 and tr.shape[2] == 5
    assert np.all(np.diff(tr.astype(np.int64), axis=2) >= 0)
    ra = a.run(200, 100, 1.0)
    rb = b.run(200, 100, 1.0)
    assert np.array_equal(ra[2], rb[2])
    assert np.array_equal(a.weights_fx(450000), b.weights_fx(450000))


@pytest.mark.parametrize("persistent", [True, False])
def test_autotune_restores_state(persistent):
    """The autotuner's trial steps leave the simulation exactly as it was."""
    ref = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    sim = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    sim.set_persistent(persistent)
    a0 = ref.run(150, 100, 1.0)
    b0 = sim.run(150, 100, 1.0)
    us = sim.autotune(20)
    assert us > 0
    a = ref.run(250, 100, 1.0)
    b = sim.run(250, 100, 1.0)
    assert np.array_equal(a0[2], b0[2])
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    assert np.array_equal(ref.weights_fx(450000), sim.weights_fx(450000))
    assert sim.elapsed_simulation() == ref.elapsed_simulation() == 400


def test_stimulus_parity():
    """Firing and current stimulus on a noisy network, including duplicate
    current entries (the last one wins, src/nemo/cpu/Simulation.cpp:160-163)."""
    sp = nb.Simulation(nb.example_random(1000, 100, 20, False), nb.Configuration())
    so = O.Simulation(O.example_random(1000, 100, 20, False), O.Configuration())
    rng = np.random.default_rng(3)
    for t in range(300):
        fstim = rng.choice(1000, 5, replace=False).tolist() if t % 3 == 0 else None
        istim = [(int(i), float(v)) for i, v in zip(rng.choice(1000, 8), rng.normal(0, 20, 8))] if t % 5 == 0 else None
        if istim:
            istim.append((istim[0][0], 7.5))
        assert sp.step(fstim, istim) == so.step(fstim, istim)


@pytest.mark.parametrize("reward", [1.0, 0.8, 0.9])
def test_stdp_analytic(reward):
    """testStdp (src/test/stdp.cpp:243-265) plus every weight equal to the oracle's"""
    assert kat.stdp_analytic(nb, reward) == kat.stdp_analytic(O, reward)


# ---------------------------------------------------------------------------
# errors (src/test/stdp.cpp:291-355, src/nemo/nemo.cpp:109-134)


def test_apply_stdp_without_stdp_fails():
    sim = nb.Simulation(nets.create_ring(nb, nb.Network(), 10, 0, True), nb.Configuration())
    sim.step()
    with pytest.raises(nb.NemoError) as e:
        sim.apply_stdp(1.0)
    assert e.value.code == 9


@pytest.mark.parametrize("stdp", [False, True])
def test_dynamic_window_length(stdp):
    """testInvalidDynamicLength: delay 34 + postfire 31 > 64 fails only with STDP."""
    conf = nb.Configuration()
    if stdp:
        pre = [np.exp(-dt / 31.0) for dt in range(31)]
        conf.set_stdp_function(pre, pre, 0.01, 1.0, -0.01, -1.0)
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, 0, *([0.0] * 7))
    net.add_neuron(iz, 1, *([0.0] * 7))
    net.add_synapse(0, 1, 34, 1.0, stdp)
    if stdp:
        with pytest.raises(nb.NemoError):
            nb.Simulation(net, conf)
    else:
        nb.Simulation(net, conf).step()


def test_literal_c2_delays_are_rejected():
    """The benchmark network with its literal 1-64 ms delays and the 20 ms
    post-fire window: max delay + |post| > 64 is rejected at creation
    (src/nemo/StdpFunction.cpp:51-60); 44 is the largest accepted."""
    with pytest.raises(nb.NemoError):
        nb.Simulation(nb.example_random(1000, 50, 64, True), nets.standard_stdp(nb))
    nb.Simulation(nb.example_random(1000, 50, 44, True), nets.standard_stdp(nb)).step()


def test_invalid_target_fails():
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, 0, *nets.exc_neuron_args())
    net.add_synapse(0, 5, 1, 1.0, False)
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, nb.Configuration())
    assert e.value.code == 6


def test_cpu_backend_is_not_provided():
    net = nets.create_ring(nb, nb.Network(), 10)
    conf = nb.Configuration()
    conf.set_cpu_backend()
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, conf)
    assert e.value.code == 5


def test_max_delay_64_delivers_nothing():
    """With STDP off a maximum delay of exactly 64 makes the reference's
    validSpikes mask zero on x86-64 (src/nemo/cpu/Simulation.cpp:263)."""
    def build(mod):
        net = nets.create_ring(mod, mod.Network(), 100, delay=1)
        net.add_synapse(0, 50, 64, 1000.0, False)
        return net
    sp = nb.Simulation(build(nb), nb.Configuration())
    so = O.Simulation(build(O), O.Configuration())
    assert sp.step([0]) == so.step([0]) == [0]
    for _ in range(200):
        assert sp.step() == so.step() == []
