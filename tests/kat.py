"""The reference's known-answer tests, written once against the shared
Network/Configuration/Simulation interface so that they run on the oracle
(tests/test_oracle_kat.py, CPU) and on the B200 backend
(tests/test_parity_gpu.py).  Each cites the reference test it restates."""
from __future__ import annotations

import numpy as np

from tests import nets

f32 = np.float32


def ring(mod, ncount, delay):
    """runRing (src/test/test.cpp:300-325)"""
    sim = mod.Simulation(nets.create_ring(mod, mod.Network(), ncount, delay=delay), mod.Configuration())
    assert sim.step([0]) == [0]
    for ms in range(1, ncount * 5 // 2):
        fired = sim.step()
        if delay == 1:
            assert fired == [ms % ncount], (ms, fired)
        elif ms % delay == 0:
            assert fired == [(ms // delay) % ncount], (ms, fired)
        else:
            assert fired == [], (ms, fired)


def double_ring(mod):
    """runDoubleRing (src/test/test.cpp:328-362)"""
    ncount = 512
    net = mod.Network()
    nets.create_ring(mod, net, ncount, 0, False, 1, 1)
    nets.create_ring(mod, net, ncount, ncount, False, 1, 2)
    sim = mod.Simulation(net, mod.Configuration())
    sim.step([0, ncount])
    for ms in range(1, ncount * 5 // 2):
        fired = sim.step()
        if ms % 2 == 0:
            assert fired == [ms % ncount, ncount + (ms // 2) % ncount]
        else:
            assert fired == [ms % ncount]


def firing_stimulus(mod):
    """testFiringStimulus (src/test/test.cpp:202-238): fired == stimulated."""
    ncount = 3000
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, np.arange(ncount, dtype=np.uint32), *nets.exc_neuron_args())
    sim = mod.Simulation(net, mod.Configuration())
    rng = np.random.default_rng(0)
    for _ in range(1000):
        fstim = np.flatnonzero(rng.random(ncount) < 10 / ncount).tolist()
        assert sorted(sim.step(fstim)) == sorted(fstim)


def current_stimulus(mod):
    """testCurrentStimulus (src/test/test.cpp:244-268)"""
    ncount = 1500
    sim = mod.Simulation(nets.create_ring(mod, mod.Network(), ncount), mod.Configuration())
    sim.step(istim=[(5, 0.001), (8, 0.001), (0, 1000.0), (100, 0.001), (1, 0.001)])
    for ms in range(1, ncount * 2):
        assert sim.step() == [ms % ncount]


def invalid_current_stimulus(mod):
    """testInvalidCurrentStimulus (src/test/test.cpp:271-284)"""
    ncount = 1000
    sim = mod.Simulation(nets.create_ring(mod, mod.Network(), ncount), mod.Configuration())
    sim.step()
    sim.step()
    try:
        sim.step(istim=[(ncount + 1, 0.5)])
    except mod.NemoError as e:
        assert e.code == 6
    else:
        raise AssertionError("invalid current stimulus accepted")


def saturation_network(mod):
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


def fixed_point_saturation(mod):
    """testFixedPointSaturation (src/test/test.cpp:414-467); returns u of
    (ref, weak, saturated) outputs."""
    sim = mod.Simulation(saturation_network(mod), mod.Configuration())
    assert len(sim.step([0, 1])) == 2
    assert len(sim.step()) == 3
    u_ref, u_weak, u_sat = (sim.get_neuron_state(k, 0) for k in (3, 4, 2))
    assert abs(u_ref - u_weak) > 1e-5
    assert abs(u_ref - u_sat) < 1e-5
    return [u_ref, u_weak, u_sat]


def non_contiguous_indices(mod, n0, nstep):
    """testNonContigousNeuronIndices (src/test/test.cpp:517-547)"""
    ncount = 1000
    s0 = mod.Simulation(nets.create_ring(mod, mod.Network(), ncount, 0, False, nstep), mod.Configuration())
    s1 = mod.Simulation(nets.create_ring(mod, mod.Network(), ncount, n0, False, nstep), mod.Configuration())
    assert s0.step([0]) == [0]
    assert s1.step([n0]) == [n0]
    for _ in range(1, 2000):
        a, b = s0.step(), s1.step()
        assert len(a) == len(b) == 1 and a[0] == b[0] - n0


def type_mixture_network(mod, iz_first):
    net = mod.Network()
    if iz_first:
        nets.create_ring(mod, net, 1024)
    ps = net.add_neuron_type("PoissonSource")
    net.add_neuron(ps, np.arange(1024, 1024 + 1000, dtype=np.uint32), 0.001)
    if not iz_first:
        nets.create_ring(mod, net, 1024)
    return net


def neuron_type_mixture(mod, iz_first):
    """testNeuronTypeMixture (src/test/test.cpp:369-410)"""
    sim = mod.Simulation(type_mixture_network(mod, iz_first), mod.Configuration())
    stream = []
    for ms in range(1000):
        fired = sorted(sim.step([0] if ms == 0 else None))
        assert fired[0] == ms % 1024
        assert all(f >= 1024 for f in fired[1:])
        stream.append(fired)
    return stream


def poisson_rate(mod, duration=10000, others=False):
    """testRate (src/test/PoissonSource.cpp:11-31)"""
    net = mod.Network()
    if others:
        nets.create_ring(mod, net, 1024, 1)
    ps = net.add_neuron_type("PoissonSource")
    net.add_neuron(ps, 0, 0.010)
    sim = mod.Simulation(net, mod.Configuration())
    nfired = sum(len(sim.step()) for _ in range(duration))
    expected = int(duration * 0.010)
    assert nfired > 0 and abs(nfired - expected) < 2 * expected
    return nfired


GROUP = 2 * 768
INIT_W = 5.0


def stdp_analytic_network(mod):
    """construct() of src/test/stdp.cpp:121-168 without noise connections"""
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")
    r = f32(0.5)
    b = f32(f32(0.25) - f32(0.05) * r)
    v = f32(-65.0)
    for g in range(2):
        net.add_neuron(iz, np.arange(g * GROUP, (g + 1) * GROUP, dtype=np.uint32),
                       f32(f32(0.02) + f32(0.08) * r), b, v, 2.0, 0.0, f32(b * v), v)
    loc = np.arange(GROUP, dtype=np.uint32)
    net.add_synapse(loc, GROUP + loc, 1 + loc % 20, np.full(GROUP, INIT_W, f32), np.ones(GROUP, np.uint8))
    return net


def stdp_analytic(mod, reward, epochs=4):
    """testStdp (src/test/stdp.cpp:243-265): after each epoch every plastic
    synapse must have changed by epoch * reward * dw(dt) (within 0.001 %).
    Returns the weights of every synapse after each epoch."""
    sim = mod.Simulation(stdp_analytic_network(mod), nets.stdp_test_configuration(mod))
    history = []
    for epoch in range(1, epochs + 1):
        for ms in range(100):
            fstim = None
            if ms == 10:
                fstim = list(range(GROUP))
            elif ms == 20:
                fstim = list(range(GROUP, 2 * GROUP))
            sim.step(fstim)
        sim.apply_stdp(reward)
        ws = []
        for local in range(GROUP):
            sid = sim.get_synapses_from(local)[0]
            d = sim.get_synapse_delay(sid)
            assert d == 1 + local % 20
            assert sim.get_synapse_plastic(sid)
            assert sim.get_synapse_target(sid) == GROUP + local
            dt = -(10 - d)
            dw = (-0.8 * np.exp(-(dt - 1) / 20.0)) if dt > 0 else (1.0 * np.exp(dt / 20.0))
            expect = INIT_W + epoch * reward * dw
            got = sim.get_synapse_weight(sid)
            assert abs(got - expect) <= 1e-5 * abs(expect), (local, got, expect)
            ws.append(got)
        history.append(ws)
    return history


def input_network(mod, ncount, izhikevich):
    """addNeurons of src/test/Input.cpp:9-22: Input neurons 0..ncount-1 (no
    parameters, no state), optionally as many Izhikevich neurons after them."""
    net = mod.Network()
    inp = net.add_neuron_type("Input")
    net.add_neuron(inp, np.arange(ncount, dtype=np.uint32))
    if izhikevich:
        iz = net.add_neuron_type("Izhikevich")
        net.add_neuron(iz, np.arange(ncount, 2 * ncount, dtype=np.uint32),
                       0.02, 0.2, -65.0, 8.0, 0.0, f32(0.2) * f32(-65.0), -65.0)
    return net


def input_create(mod, ncount, izhikevich):
    """create (src/test/Input.cpp:29-37): a network of Input neurons steps."""
    sim = mod.Simulation(input_network(mod, ncount, izhikevich), mod.Configuration())
    assert sim.step() == []


def input_simple(mod, ncount, izhikevich, steps=1000, seed=0):
    """simple (src/test/Input.cpp:41-63): Input neurons fire exactly when
    stimulated, in stimulus order.  Returns the fire stream."""
    sim = mod.Simulation(input_network(mod, ncount, izhikevich), mod.Configuration())
    rng = np.random.default_rng(seed)
    stream = []
    for _ in range(steps):
        p = 0.5 * rng.random()
        fstim = np.flatnonzero(rng.random(ncount) < p).tolist()
        fired = sim.step(fstim)
        assert fired == fstim
        stream.append(fired)
    return stream


def clamp_network(mod):
    """Four plastic synapses whose weights start outside the STDP limits of
    clamp_configuration (above the excitatory maximum, below the excitatory
    minimum, beyond the inhibitory maximum, inside the inhibitory minimum),
    a plastic zero weight, and one static synapse out of range."""
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, np.arange(8, dtype=np.uint32), *nets.exc_neuron_args())
    ws = [15.0, 0.5, -15.0, -0.5, 0.0, 15.0]
    plastic = [1, 1, 1, 1, 1, 0]
    net.add_synapse(np.zeros(6, np.uint32), np.arange(1, 7, dtype=np.uint32), np.ones(6, np.uint32),
                    np.array(ws, f32), np.array(plastic, np.uint8))
    return net


def clamp_configuration(mod):
    """STDP limits E [2, 10], I [-2, -10] (setStdpFunction's six-argument
    form, src/nemo/Configuration.cpp:92-100)"""
    conf = mod.Configuration()
    pre = np.array([f32(0.1) * np.exp(f32(-dt) / f32(20.0), dtype=f32) for dt in range(1, 21)], f32)
    post = np.array([f32(-0.12) * np.exp(f32(-dt) / f32(20.0), dtype=f32) for dt in range(1, 21)], f32)
    conf.set_stdp_function(pre, post, 2.0, 10.0, -2.0, -10.0)
    return conf


def first_call_clamp(mod, reward):
    """The first applyStdp visits every plastic synapse and clamps weights
    that start outside the limits even where nothing accumulated
    (ConnectivityMatrix::applyStdp, src/nemo/ConnectivityMatrix.cpp:241-294;
    StdpProcess::updatedWeight, src/nemo/StdpProcess.cpp:128-138); a zero
    weight stays zero and static synapses are not touched.  Returns the
    weights after the call."""
    sim = mod.Simulation(clamp_network(mod), clamp_configuration(mod))
    sim.step()
    sim.apply_stdp(reward)
    ws = [sim.get_synapse_weight(sim.get_synapses_from(0)[k]) for k in range(6)]
    assert ws == [10.0, 2.0, -10.0, -2.0, 0.0, 15.0], ws
    return ws


def zero_reward_clears(mod):
    """applyStdp(0) clears the accumulators and leaves the weights (all
    within limits) unchanged: an applyStdp(1.0) straight after it changes
    nothing, while on a twin simulation without it the same call changes
    weights (src/nemo/ConnectivityMatrix.cpp:251-259).  Returns the weights
    of the twin after 50 more steps and applyStdp(0.8)."""
    def make():
        s = mod.Simulation(stdp_analytic_network(mod), nets.stdp_test_configuration(mod))
        for ms in range(100):
            fstim = list(range(GROUP)) if ms == 10 else list(range(GROUP, 2 * GROUP)) if ms == 20 else None
            s.step(fstim)
        return s

    def weights(s):
        return [s.get_synapse_weight(s.get_synapses_from(k)[0]) for k in range(GROUP)]

    cleared, twin = make(), make()
    cleared.apply_stdp(0.0)
    assert weights(cleared) == [INIT_W] * GROUP
    cleared.apply_stdp(1.0)
    assert weights(cleared) == [INIT_W] * GROUP
    twin.apply_stdp(1.0)
    assert weights(twin) != [INIT_W] * GROUP
    for s in (cleared, twin):
        for ms in range(50):
            s.step(list(range(GROUP)) if ms == 10 else list(range(GROUP, 2 * GROUP)) if ms == 20 else None)
        s.apply_stdp(0.8)
    return weights(cleared), weights(twin)


FX = float(1 << 20)


def fx_round_trip(w):
    """fx_toFloat(fx_toFix(w)) (src/nemo/fixedpoint.cpp:17-36): truncation
    to Q11.20 and back, in float32."""
    return float(np.float32(int(np.float32(w) * np.float32(FX))) / np.float32(FX))


def expected_synapses(src, tgt, dly, w, pl):
    """The network's synapse ids (source << 32 | index by insertion order per
    source, src/nemo/NetworkImpl.cpp:105-130) with their target, delay,
    fixed-point rounded weight and plasticity."""
    out, count = {}, {}
    for s, t, d, x, p in zip(src.tolist(), tgt.tolist(), dly.tolist(), w.tolist(), pl.tolist()):
        i = count.get(s, 0)
        count[s] = i + 1
        out.setdefault(s, []).append(((s << 32) | i, t, d, fx_round_trip(x), bool(p)))
    return out


def get_synapses(mod, stdp):
    """testGetSynapses (src/test/test.cpp:562-603): the simulation holds the
    network's synapses -- the same ids per source, targets, delays,
    plasticity and (fixed-point rounded) weights -- on a random network and
    on a ring whose indices start at 10^6.  Returns the simulation's
    (id, target, delay, weight, plastic) tuples."""
    import oracle as O
    conf = nets.standard_stdp(mod) if stdp else mod.Configuration()
    ring = np.arange(1000000, 1001500, dtype=np.uint32)
    cases = [(mod.example_random(300, 50, 20, stdp), expected_synapses(*O.example_random(300, 50, 20, stdp).synapses())),
             (nets.create_ring(mod, mod.Network(), 1500, 1000000),
              expected_synapses(ring, np.roll(ring, -1), np.ones(1500, np.uint32), np.full(1500, 1000.0, f32),
                                np.zeros(1500, np.uint8)))]
    out = []
    for net, expect in cases:
        sim = mod.Simulation(net, conf)
        sim.step()
        for src, syn in sorted(expect.items())[::3]:
            assert list(sim.get_synapses_from(src)) == [x[0] for x in syn], src
            for i, t, d, w, p in syn:
                got = (i, sim.get_synapse_target(i), sim.get_synapse_delay(i), sim.get_synapse_weight(i),
                       bool(sim.get_synapse_plastic(i)))
                assert got == (i, t, d, w, p), (got, (i, t, d, w, p))
                out.append(got)
    return out


def write_only_synapses(mod):
    """testWriteOnlySynapses (src/test/test.cpp:605-624)"""
    conf = mod.Configuration()
    conf.set_write_only_synapses()
    sim = mod.Simulation(nets.create_ring(mod, mod.Network(), 10, 0, True), conf)
    sim.step()
    for query in (lambda: sim.get_synapses_from(0), lambda: sim.get_synapse_weight((1 << 32) | 0)):
        try:
            query()
        except mod.NemoError:
            pass
        else:
            raise AssertionError("write-only synapses were read")


def synapses_from_unconnected_neuron(mod):
    """testGetSynapsesFromUnconnectedNeuron (src/test/test.cpp:626-655)"""
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")
    for n in range(4):
        net.add_neuron(iz, n, 0.1, 0.2, 0.3, 0.4, 0.7, 0.5, 0.6)
    sim = mod.Simulation(net, mod.Configuration())
    sim.step()
    try:
        sim.get_synapses_from(4)
    except mod.NemoError:
        pass
    else:
        raise AssertionError("synapses of a non-existing neuron")
    assert list(sim.get_synapses_from(3)) == []


def high_firing(mod, steps=1000):
    """testHighFiring (src/test/test.cpp:697-736): every neuron stimulated
    to fire every step (1024 neurons x 1000 synapses, delays 1-32): every
    delivery group of every source is pending at once.  Returns the state."""
    n = 1024
    sim = mod.Simulation(mod.example_random(n, 1000, 32, False), mod.Configuration())
    everyone = list(range(n))
    for _ in range(steps):
        assert sim.step(everyone) == everyone
    return sim.type_state(0, 2, n)


def vprobe(mod):
    """testVProbe (src/test/test.cpp:738-753): the membrane potential of a
    new simulation is the one it was given."""
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")
    v0 = -65.0
    net.add_neuron(iz, 0, 0.02, 0.2, -65.0 + 15.0 * 0.25, 8.0 - 6.0 * 0.25, 5.0, 0.2 * -65.0, v0)
    sim = mod.Simulation(net, mod.Configuration())
    assert sim.get_membrane_potential(0) == v0


def stdp_with_all_static(mod):
    """testStdpWithAllStatic (src/test/test.cpp:666-680): STDP configured
    but no plastic synapse; applyStdp is accepted and changes nothing."""
    net = mod.example_random(1000, 1000, 1, False)
    sim = mod.Simulation(net, nets.standard_stdp(mod))
    stream = []
    for _ in range(2):
        for _ in range(300):
            stream.append(sim.step())
        sim.apply_stdp(1.0)
    return stream


def set_neuron_network(mod):
    """testSetNeuron, the network half (src/test/test.cpp:769-835):
    setters and getters of a neuron before a simulation exists, and their
    index and variable errors.  Arguments in the Izhikevich plugin order
    (a, b, c, d, sigma | u, v)."""
    a, b, c, d = f32(0.02), f32(0.2), f32(-65.0 + 15.0 * 0.25), f32(8.0 - 6.0 * 0.25)
    v = f32(-65.0)
    u, sigma, e = f32(b * v), f32(5.0), f32(0.1)
    net = mod.Network()
    iz = net.add_neuron_type("Izhikevich")

    def fails(f):
        try:
            f()
        except mod.NemoError:
            return True
        return False
    assert fails(lambda: net.set_neuron(0, a, b, c, d, sigma, u, v))
    net.add_neuron(iz, 0, a, b, f32(c - f32(0.1)), d, sigma, u, f32(v - f32(1.0)))
    assert fails(lambda: net.get_neuron_parameter(1, 0)) and fails(lambda: net.get_neuron_state(1, 0))
    assert fails(lambda: net.get_neuron_parameter(0, 5)) and fails(lambda: net.get_neuron_state(0, 2))
    args = [f32(x - e) for x in (a, b, c, d, sigma, u, v)]
    net.set_neuron(0, *args)
    assert [net.get_neuron_parameter(0, k) for k in range(5)] + [net.get_neuron_state(0, k) for k in range(2)] \
        == [float(x) for x in args]
    for k, x in enumerate((a, b, c, d, sigma)):
        net.set_neuron_parameter(0, k, x)
        assert net.get_neuron_parameter(0, k) == float(x)
    for k, x in enumerate((u, v)):
        net.set_neuron_state(0, k, x)
        assert net.get_neuron_state(0, k) == float(x)
    assert fails(lambda: net.set_neuron_parameter(1, 0, 0.0)) and fails(lambda: net.set_neuron_state(1, 0, 0.0))
    assert fails(lambda: net.set_neuron_parameter(0, 5, 0.0)) and fails(lambda: net.set_neuron_state(0, 2, 0.0))
    return net, (a, b, c, d, sigma, u, v, e)


def set_neuron_simulation(mod):
    """testSetNeuron, the simulation half (src/test/test.cpp:837-963):
    setters during a run take effect without being overwritten, parameters
    stay and state evolves, errors for invalid indices, a changed c that the
    neuron does not use leaves the run unchanged, setting the state does
    not copy it twice, and a potential set before the first step is the one
    simulated.  Returns the membrane potentials it observed."""
    a, b, c, d = f32(0.02), f32(0.2), f32(-65.0 + 15.0 * 0.25), f32(8.0 - 6.0 * 0.25)
    v = f32(-65.0)
    u, sigma, e = f32(b * v), f32(5.0), f32(0.1)
    # the network the network half leaves (set_neuron_network)
    net = mod.Network()
    net.add_neuron(net.add_neuron_type("Izhikevich"), 0, a, b, c, d, sigma, u, v)
    conf = mod.Configuration()

    def fails(f):
        try:
            f()
        except mod.NemoError:
            return True
        return False
    seen = []
    sim = mod.Simulation(net, conf)
    sim.step()
    sim.set_neuron_state(0, 0, f32(u - e))
    assert sim.get_neuron_state(0, 0) == float(f32(u - e))
    sim.set_neuron_state(0, 1, f32(v - e))
    assert sim.get_neuron_state(0, 1) == float(f32(v - e))
    u0, v0 = sim.get_neuron_state(0, 0), sim.get_neuron_state(0, 1)
    for k, x in enumerate((a, b, c, d, sigma)):
        sim.set_neuron_parameter(0, k, f32(x - e))
        assert sim.get_neuron_parameter(0, k) == float(f32(x - e))
    sim.step()
    for k, x in enumerate((a, b, c, d, sigma)):
        assert sim.get_neuron_parameter(0, k) == float(f32(x - e))
    assert sim.get_neuron_state(0, 0) != u0 and sim.get_neuron_state(0, 1) != v0
    seen += [sim.get_neuron_state(0, 0), sim.get_neuron_state(0, 1)]
    for f in (lambda: sim.set_neuron_parameter(1, 0, 0.0), lambda: sim.set_neuron_state(1, 0, 0.0),
              lambda: sim.get_neuron_parameter(1, 0), lambda: sim.get_neuron_state(1, 0),
              lambda: sim.set_neuron_parameter(0, 5, 0.0), lambda: sim.set_neuron_state(0, 2, 0.0),
              lambda: sim.get_neuron_parameter(0, 5), lambda: sim.get_neuron_state(0, 2)):
        assert fails(f)
    del sim

    sim = mod.Simulation(net, conf)
    sim.step()
    v0 = sim.get_membrane_potential(0)
    del sim
    sim = mod.Simulation(net, conf)
    assert sim.get_neuron_state(0, 0) == float(u) and sim.get_neuron_state(0, 1) == float(v)
    sim.set_neuron(0, a, b, f32(c + f32(1.0)), d, sigma, u, v)
    sim.step()
    assert v0 == sim.get_membrane_potential(0)
    assert [sim.get_neuron_parameter(0, k) for k in range(5)] == [float(x) for x in (a, b, f32(c + f32(1.0)), d, sigma)]
    seen.append(v0)
    del sim

    net0 = mod.Network()
    iz = net0.add_neuron_type("Izhikevich")
    net0.add_neuron(iz, 0, a, b, c, d, 0.0, u, v)
    sim0 = mod.Simulation(net0, conf)
    sim0.step()
    sim0.step()
    sim1 = mod.Simulation(net0, conf)
    sim1.step()
    sim1.set_neuron(0, a, b, c, d, 0.0, u, v)
    sim1.step()
    sim1.step()
    assert sim0.get_membrane_potential(0) == sim1.get_membrane_potential(0)
    seen.append(sim1.get_membrane_potential(0))

    net1 = mod.Network()
    iz = net1.add_neuron_type("Izhikevich")
    net1.add_neuron(iz, 0, a, b, c, d, sigma, u, f32(v - f32(1.0)))
    sim = mod.Simulation(net1, conf)
    sim.set_neuron(0, a, b, c, d, sigma, u, v)
    assert sim.get_membrane_potential(0) == float(v)
    sim.step()
    assert sim.get_membrane_potential(0) == v0
    return seen


def izhikevich_rs_no_parameters(mod):
    """testNoParamNeuronType (src/test/test.cpp:980-1000): IzhikevichRS
    neurons take only their state (u, v); 100 steps keep it finite.
    Returns (u, v) of every neuron."""
    net = mod.Network()
    rs = net.add_neuron_type("IzhikevichRS")
    net.add_neuron(rs, np.arange(1000, dtype=np.uint32), -13.0, -65.0)
    sim = mod.Simulation(net, mod.Configuration())
    for _ in range(100):
        sim.step()
        u, v = sim.get_neuron_state(100, 0), sim.get_neuron_state(100, 1)
        assert np.isfinite(u) and np.isfinite(v)
    return sim.type_state(rs, 2, 1000)


def izhikevich_rs_network(mod, steps=500, seed=11, resident=True):
    """A connected IzhikevichRS network (1000 neurons, 50 random synapses
    each, mixed signs, delays 1-10) driven by a firing stimulus every 5
    steps and a current stimulus every 7.  Returns the fire stream and the
    final state."""
    rng = np.random.default_rng(seed)
    n = 1000
    net = mod.Network()
    rs = net.add_neuron_type("IzhikevichRS")
    net.add_neuron(rs, np.arange(n, dtype=np.uint32), -13.0, -65.0)
    src = np.repeat(np.arange(n, dtype=np.uint32), 50)
    tgt = rng.integers(0, n, len(src)).astype(np.uint32)
    w = np.where(rng.random(len(src)) < 0.8, 6.0 * rng.random(len(src)), -8.0 * rng.random(len(src))).astype(f32)
    dly = rng.integers(1, 11, len(src)).astype(np.uint32)
    net.add_synapse(src, tgt, dly, w, np.zeros(len(src), np.uint8))
    sim = mod.Simulation(net, mod.Configuration())
    if not resident:
        sim.set_resident_step(0)
    stream = []
    for t in range(steps):
        fstim = rng.choice(n, 20, replace=False).tolist() if t % 5 == 0 else None
        istim = [(int(i), 12.0) for i in rng.choice(n, 30, replace=False)] if t % 7 == 0 else None
        stream.append(sim.step(fstim, istim))
    return stream, sim.type_state(rs, 2, n)


def close(a, b, percent=0.001):
    """BOOST_REQUIRE_CLOSE: |a - b| within `percent` % of both a and b"""
    d = abs(float(a) - float(b))
    return d <= percent / 100 * abs(float(a)) and d <= percent / 100 * abs(float(b))


def oscillator_network(mod):
    """OscillatorNetwork (src/test/Kuramoto.cpp:11-34)"""
    net = mod.Network()
    return net, net.add_neuron_type("Kuramoto")


def kuramoto_init(mod):
    """testInit (src/test/Kuramoto.cpp:42-61)"""
    net, k = oscillator_network(mod)
    net.add_neuron(k, 0, 0.1, 0.0)
    sim = mod.Simulation(net, mod.Configuration())
    assert sim.get_neuron_state(0, 0) == 0.0
    sim.step()
    assert close(sim.get_neuron_state(0, 0), f32(0.0) + f32(0.1))


def kuramoto_uncoupled(mod):
    """testUncoupled (src/test/Kuramoto.cpp:65-86)"""
    net, k = oscillator_network(mod)
    n, freq = 1200, f32(0.1)
    net.add_neuron(k, np.arange(n, dtype=np.uint32), freq, 0.0)
    sim = mod.Simulation(net, mod.Configuration())
    phase = f32(0.0)
    for _ in range(1000):
        sim.step()
        phase = np.fmod(f32(phase + freq), f32(2 * np.pi))
        assert close(sim.get_neuron_state(n // 2, 0), phase)


def kuramoto_simple_coupled(mod):
    """testSimpleCoupled (src/test/Kuramoto.cpp:90-122).  Returns both
    phases after every step."""
    net, k = oscillator_network(mod)
    freq, phase = [f32(0.1), f32(0.1)], [f32(0.0), f32(1.57)]
    net.add_neuron(k, 0, freq[0], phase[0])
    net.add_neuron(k, 1, freq[1], phase[1])
    net.add_synapse(0, 1, 1, 1.0, False)
    sim = mod.Simulation(net, mod.Configuration())
    seen = []
    for _ in range(100):
        sim.step()
        k1 = f32(freq[0] + np.sin(phase[0] - phase[1]))
        k2 = f32(freq[0] + np.sin(phase[0] - f32(phase[1] + f32(0.5) * k1)))
        k3 = f32(freq[0] + np.sin(phase[0] - f32(phase[1] + f32(0.5) * k2)))
        k4 = f32(freq[0] + np.sin(phase[0] - f32(phase[1] + k3)))
        phase[1] = f32(phase[1] + f32(f32(k1 + f32(2.0) * k2 + f32(2.0) * k3 + k4) / f32(6.0)))
        phase[0] = f32(phase[0] + freq[0])
        for i in range(2):
            phase[i] = np.fmod(phase[i], f32(2 * np.pi))
            assert close(sim.get_neuron_state(i, 0), phase[i]), (i, sim.get_neuron_state(i, 0), phase[i])
        seen.append([sim.get_neuron_state(0, 0), sim.get_neuron_state(1, 0)])
    return np.array(seen, np.float32)


def kuramoto_n_to_1(mod, ncount, noise):
    """testNto1 (src/test/Kuramoto.cpp:126-185): one oscillator driven by
    ncount others of strength 1/ncount (with zero-strength couplings among
    the others when `noise`).  Returns the driven phase after every step."""
    net, k = oscillator_network(mod)
    freq, strength = f32(0.1), f32(1.0 / ncount)
    phase0 = phaseN = f32(0.0)
    net.add_neuron(k, 0, freq, phase0)
    for n in range(ncount):
        net.add_neuron(k, n + 1, freq, phaseN)
        net.add_synapse(n + 1, 0, 1, strength, False)
        if noise:
            tgts = [t for t in range(1, ncount) if t != n + 1]
            if tgts:
                net.add_synapse(np.full(len(tgts), n + 1, np.uint32), np.array(tgts, np.uint32),
                                np.ones(len(tgts), np.uint32), np.zeros(len(tgts), f32), np.zeros(len(tgts), np.uint8))
    sim = mod.Simulation(net, mod.Configuration())
    seen = []
    for _ in range(50):
        sim.step()
        w = f32(ncount) * strength
        k1 = f32(freq + w * np.sin(f32(phaseN - phase0), dtype=f32))
        k2 = f32(freq + w * np.sin(f32(phaseN - f32(phase0 + f32(0.5) * k1)), dtype=f32))
        k3 = f32(freq + w * np.sin(f32(phaseN - f32(phase0 + f32(0.5) * k2)), dtype=f32))
        k4 = f32(freq + w * np.sin(f32(phaseN - f32(phase0 + k3)), dtype=f32))
        phase0 = f32(phase0 + f32(f32(k1 + f32(2.0) * k2 + f32(2.0) * k3 + k4) / f32(6.0)))
        phase0 = np.fmod(phase0, f32(2 * np.pi))
        phaseN = np.fmod(f32(phaseN + freq), f32(2 * np.pi))
        assert close(sim.get_neuron_state(0, 0), phase0), (sim.get_neuron_state(0, 0), phase0)
        for n in range(0, ncount, max(1, ncount // 7)):
            assert close(sim.get_neuron_state(n + 1, 0), phaseN)
        seen.append(sim.get_neuron_state(0, 0))
    return np.array(seen, np.float32)


def kuramoto_with_stdp_fails(mod):
    """A type that reads its sources cannot coexist with STDP
    (src/nemo/construction/RCM.cpp:90-98): NEMO_API_UNSUPPORTED"""
    net, k = oscillator_network(mod)
    net.add_neuron(k, 0, 0.1, 0.0)
    net.add_neuron(k, 1, 0.1, 1.0)
    net.add_synapse(0, 1, 1, 1.0, True)
    try:
        mod.Simulation(net, nets.standard_stdp(mod))
    except mod.NemoError as e:
        assert "does not support a mix of STDP" in str(e)
        return e.code
    raise AssertionError("STDP with a reverse-matrix type accepted")


def kuramoto_random(mod, ncount=2048, scount=32, steps=1000, seed=5):
    """The reference's example oscillator network (src/examples/
    kuramoto.cpp:49-68): frequencies U(0, 0.2), phases U(0, 2 pi), scount
    outgoing couplings of strength 0.001 and lag 1 to uniform targets; here
    with lags 1-20 as well.  Seeded numpy draws stand in for the Boost
    generator.  Returns the phases after `steps` steps."""
    rng = np.random.default_rng(seed)
    net, k = oscillator_network(mod)
    freq = rng.uniform(0.0, 0.2, ncount).astype(f32)
    phase = rng.uniform(0.0, 2 * np.pi, ncount).astype(f32)
    net.add_neuron(k, np.arange(ncount, dtype=np.uint32), freq, phase)
    src = np.repeat(np.arange(ncount, dtype=np.uint32), scount)
    tgt = rng.integers(0, ncount, len(src)).astype(np.uint32)
    lag = rng.integers(1, 21, len(src)).astype(np.uint32)
    net.add_synapse(src, tgt, lag, np.full(len(src), 0.001, f32), np.zeros(len(src), np.uint8))
    sim = mod.Simulation(net, mod.Configuration())
    for _ in range(steps):
        assert sim.step() == []
    return sim.type_state(k, 1, ncount)[0]
