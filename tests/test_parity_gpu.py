"""Parity of the B200 backend (through its C ABI) with the CPU oracle and with
the reference's own known-answer tests (src/test/test.cpp, src/test/stdp.cpp,
src/test/PoissonSource.cpp).  The bar is bit-exactness: identical fire
streams (cycle, neuron id), identical fp32 neuron state (NaN compared as NaN)
and identical fixed-point weights."""
import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

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
# known-answer tests of the reference (src/test/test.cpp)

@pytest.mark.parametrize("ncount,delay", [(1000, 1), (1024, 1), (2000, 1), (4000, 1), (2000, 20)])
def test_ring(ncount, delay):
    """runRing (src/test/test.cpp:300-325)"""
    net = nets.create_ring(nb, nb.Network(), ncount, delay=delay)
    sim = nb.Simulation(net, nb.Configuration())
    assert sim.step([0]) == [0]
    for ms in range(1, ncount * 5 // 2):
        fired = sim.step()
        if delay == 1:
            assert fired == [ms % ncount], (ms, fired)
        elif ms % delay == 0:
            assert fired == [(ms // delay) % ncount], (ms, fired)
        else:
            assert fired == [], (ms, fired)


def test_double_ring():
    """runDoubleRing (src/test/test.cpp:328-362)"""
    ncount = 512
    net = nb.Network()
    nets.create_ring(nb, net, ncount, 0, False, 1, 1)
    nets.create_ring(nb, net, ncount, ncount, False, 1, 2)
    sim = nb.Simulation(net, nb.Configuration())
    sim.step([0, ncount])
    for ms in range(1, ncount * 5 // 2):
        fired = sim.step()
        if ms % 2 == 0:
            assert fired == [ms % ncount, ncount + (ms // 2) % ncount]
        else:
            assert fired == [ms % ncount]


def test_firing_stimulus():
    """testFiringStimulus (src/test/test.cpp:202-238): fired == stimulated."""
    ncount = 3000
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, np.arange(ncount, dtype=np.uint32), *nets.exc_neuron_args())
    sim = nb.Simulation(net, nb.Configuration())
    rng = np.random.default_rng(0)
    for _ in range(1000):
        fstim = np.flatnonzero(rng.random(ncount) < 10 / ncount).tolist()
        assert sorted(sim.step(fstim)) == sorted(fstim)


def test_current_stimulus():
    """testCurrentStimulus (src/test/test.cpp:244-268)"""
    ncount = 1500
    sim = nb.Simulation(nets.create_ring(nb, nb.Network(), ncount), nb.Configuration())
    istim = [(5, 0.001), (8, 0.001), (0, 1000.0), (100, 0.001), (1, 0.001)]
    sim.step(istim=istim)
    for ms in range(1, ncount * 2):
        assert sim.step() == [ms % ncount]


def test_invalid_current_stimulus():
    """testInvalidCurrentStimulus (src/test/test.cpp:271-284)"""
    ncount = 1000
    sim = nb.Simulation(nets.create_ring(nb, nb.Network(), ncount), nb.Configuration())
    sim.step()
    sim.step()
    with pytest.raises(nb.NemoError) as e:
        sim.step(istim=[(ncount + 1, 0.5)])
    assert e.value.code == 6


def test_fixed_point_saturation():
    """testFixedPointSaturation (src/test/test.cpp:414-467), also bit-exact
    against the oracle."""
    def build(mod):
        net = mod.Network()
        iz = net.add_neuron_type("Izhikevich")
        params = [0.02, 0.2, -65.0, 8.0, 0.0, -13.0, -65.0]
        for n in range(5):
            net.add_neuron(iz, n, *params)
        INPUT0, INPUT1, OUT_SAT, OUT_REF, OUT_WEAK = range(5)
        for s, t, w in [(INPUT0, OUT_REF, 1024.0), (INPUT1, OUT_REF, 1024.0), (INPUT0, OUT_WEAK, 1000.0),
                        (INPUT1, OUT_WEAK, 1000.0), (INPUT0, OUT_SAT, 1100.0), (INPUT1, OUT_SAT, 1100.0)]:
            net.add_synapse(s, t, 1, w, False)
        return net
    sims = [m.Simulation(build(m), m.Configuration()) for m in (nb, O)]
    for sim in sims:
        assert len(sim.step([0, 1])) == 2
        assert len(sim.step()) == 3
    u = [[sim.get_neuron_state(k, 0) for k in (3, 4, 2)] for sim in sims]
    u_ref, u_weak, u_sat = u[0]
    assert abs(u_ref - u_weak) > 1e-5
    assert abs(u_ref - u_sat) < 1e-5
    assert same_bits(u[0], u[1])


@pytest.mark.parametrize("n0,nstep", [(1, 1), (1000000, 1), (1, 4), (1000000, 4)])
def test_non_contiguous_indices(n0, nstep):
    """testNonContigousNeuronIndices (src/test/test.cpp:517-547)"""
    ncount = 1000
    s0 = nb.Simulation(nets.create_ring(nb, nb.Network(), ncount, 0, False, nstep), nb.Configuration())
    s1 = nb.Simulation(nets.create_ring(nb, nb.Network(), ncount, n0, False, nstep), nb.Configuration())
    f0 = s0.step([0])
    f1 = s1.step([n0])
    assert f0 == [0] and f1 == [n0]
    for _ in range(1, 2000):
        a, b = s0.step(), s1.step()
        assert len(a) == len(b) == 1 and a[0] == b[0] - n0


@pytest.mark.parametrize("iz_first", [True, False])
def test_neuron_type_mixture(iz_first):
    """testNeuronTypeMixture (src/test/test.cpp:369-410): a Poisson
    population beside a ring must not disturb it; bit-exact with the oracle."""
    def build(mod):
        net = mod.Network()
        if iz_first:
            nets.create_ring(mod, net, 1024)
        ps = net.add_neuron_type("PoissonSource")
        net.add_neuron(ps, np.arange(1024, 1024 + 1000, dtype=np.uint32), 0.001)
        if not iz_first:
            nets.create_ring(mod, net, 1024)
        return net
    sp = nb.Simulation(build(nb), nb.Configuration())
    so = O.Simulation(build(O), O.Configuration())
    for ms in range(1000):
        st = [0] if ms == 0 else None
        a = sp.step(st)
        b = so.step(st)
        assert a == b
        fired = sorted(a)
        assert fired[0] == ms % 1024
        assert all(f >= 1024 for f in fired[1:])


def test_poisson_rate():
    """testRate (src/test/PoissonSource.cpp:11-31) plus oracle parity."""
    for mod in (nb,):
        net = mod.Network()
        ps = net.add_neuron_type("PoissonSource")
        net.add_neuron(ps, 0, 0.010)
        sim = mod.Simulation(net, mod.Configuration())
        counts, _, _ = sim.run(10000)
        nfired = int(counts.sum())
        expected = int(10000 * 0.010)
        assert nfired > 0 and abs(nfired - expected) < 2 * expected


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


def test_stdp_bitexact():
    """A 2000 x 200 random network with STDP (delays 1-20, window 20+20,
    applyStdp(1.0) every 100 ms): fire stream, state and every weight."""
    sims = (nb.Simulation(nb.example_random(2000, 200, 20, True), nets.standard_stdp(nb)),
            O.Simulation(O.example_random(2000, 200, 20, True), nets.standard_stdp(O)))
    p, o = run_both(sims, 1000, stdp_period=100)
    assert_streams_equal(p, o)
    nsyn = 2000 * 200
    wp, wo = sims[0].weights_fx(nsyn), sims[1].weights_fx(nsyn)
    assert not np.array_equal(wp, O.example_random(2000, 200, 20, True).synapses()[3])  # weights did change
    assert np.array_equal(wp, wo)
    assert same_bits(sims[0].type_state(0, 2, 2000), sims[1].type_state(0, 2, 2000))


def test_stdp_inflight_compensation():
    """applyStdp between a spike's emission and its arrival: the arriving
    weight is the updated one (long delays, frequent applyStdp)."""
    sims = (nb.Simulation(nb.example_random(1500, 150, 40, True), nets.standard_stdp(nb, n=20)),
            O.Simulation(O.example_random(1500, 150, 40, True), nets.standard_stdp(O, n=20)))
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


def test_stdp_analytic():
    """testStdp (src/test/stdp.cpp:243-265): after each epoch every
    one-to-one plastic synapse must have changed by epoch*reward*dw(dt)."""
    group = 2 * 768
    init_w = 5.0

    def build(mod):
        net = mod.Network()
        iz = net.add_neuron_type("Izhikevich")
        r = f32(0.5)
        b = f32(f32(0.25) - f32(0.05) * r)
        v = f32(-65.0)
        for g in range(2):
            net.add_neuron(iz, np.arange(g * group, (g + 1) * group, dtype=np.uint32),
                           f32(f32(0.02) + f32(0.08) * r), b, v, 2.0, 0.0, f32(b * v), v)
        loc = np.arange(group, dtype=np.uint32)
        net.add_synapse(loc, group + loc, 1 + loc % 20, np.full(group, init_w, f32), np.ones(group, np.uint8))
        return net

    for reward in (1.0, 0.8):
        sims = [m.Simulation(build(m), nets.stdp_test_configuration(m)) for m in (nb, O)]
        for epoch in range(1, 5):
            for ms in range(100):
                fstim = None
                if ms == 10:
                    fstim = list(range(group))
                elif ms == 20:
                    fstim = list(range(group, 2 * group))
                a = sims[0].step(fstim)
                assert a == sims[1].step(fstim)
            for s in sims:
                s.apply_stdp(reward)
            for local in range(0, group, 37):
                sid = sims[0].get_synapses_from(local)[0]
                d = sims[0].get_synapse_delay(sid)
                assert d == 1 + local % 20
                dt = -(10 - d)
                dw = (-0.8 * np.exp(-(dt - 1) / 20.0)) if dt > 0 else (1.0 * np.exp(dt / 20.0))
                expect = init_w + epoch * reward * dw
                got = sims[0].get_synapse_weight(sid)
                assert got == pytest.approx(expect, rel=1e-5)
                assert got == sims[1].get_synapse_weight(sid)


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
