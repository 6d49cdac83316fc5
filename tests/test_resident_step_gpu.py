"""nemo_step through the resident step loop (a cooperative launch that stays
on the GPU between calls) against nemo_step with two kernel launches per
call: identical fired neurons, neuron state and weights, across stimuli of
every size, applyStdp, run(), queries, the loop's idle time-out and its
relaunch, and two simulations that alternate on one GPU."""
import time

import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

pytestmark = pytest.mark.gpu


def pair(n=2000, fanout=120, stdp=True):
    make = lambda: nb.Simulation(nb.example_random(n, fanout, 20, stdp),
                                 nets.standard_stdp(nb) if stdp else nb.Configuration())
    resident, plain = make(), make()
    plain.set_resident_step(0)
    return resident, plain


def same_state(a, b, n):
    sa = np.asarray(a.type_state(0, 2, n), np.float32).view(np.uint32)
    sb = np.asarray(b.type_state(0, 2, n), np.float32).view(np.uint32)
    return np.array_equal(sa, sb)


def script(n, steps, seed):
    """Per step: a firing stimulus and a current stimulus (or None), with
    some large ones that outgrow the staging buffer.  Firing stimuli of 1-8
    neurons cover both sides of the six that travel inside the resident
    loop's request line, and one repeats a neuron."""
    rng = np.random.default_rng(seed)
    out = []
    for t in range(steps):
        f = rng.choice(n, int(rng.integers(1, 9)), replace=False).tolist() if t % 3 == 0 else None
        i = [(int(a), float(v)) for a, v in zip(rng.choice(n, 4), rng.normal(0, 15, 4))] if t % 7 == 0 else None
        if t == 60:
            f = [5, 17, 5]
        if t in (40, 41):
            f = rng.choice(n, n // 2, replace=False).tolist()       # beyond the initial buffer
            i = [(int(a), 3.0) for a in rng.choice(n, 700)]
        out.append((f, i))
    return out


def drive(sim, plan, period, reward=1.0):
    fired = []
    for t, (f, i) in enumerate(plan):
        fired.append(list(sim.step(f, i)))
        if period and (t + 1) % period == 0:
            sim.apply_stdp(reward)
    return fired


def test_resident_step_matches_two_launch_step():
    n = 2000
    a, b = pair(n)
    plan = script(n, 400, 1)
    # one simulation at a time, so that neither waits on the other's loop
    fa = drive(a, plan, 50)
    fb = drive(b, plan, 50)
    assert fa == fb
    assert sum(map(len, fa)) > 1000
    assert same_state(a, b, n)
    assert np.array_equal(a.weights_fx(), b.weights_fx())
    assert a.elapsed_simulation() == b.elapsed_simulation() == 400
    assert a.step_events() == b.step_events()


def test_other_calls_end_the_loop_between_steps():
    """Queries, run() and setters between resident steps see the state the
    steps left, and steps after them continue the same simulation."""
    n = 2000
    a, b = pair(n)
    plan = script(n, 120, 2)
    for sim in (a, b):
        sim.trace = []
        for t, (f, i) in enumerate(plan):
            sim.trace.append(list(sim.step(f, i)))
            if t == 30:
                sim.trace.append(np.asarray(sim.type_state(0, 2, n), np.float32).tobytes())
            if t == 60:
                c, _, ids = sim.run(77, 25, 1.0)
                sim.trace.append((c.tolist(), ids.tolist()))
            if t == 90:
                sim.set_neuron_state(5, 0, 25.0)
                sim.trace.append(sim.get_membrane_potential(5))
    assert a.trace == b.trace
    assert same_state(a, b, n)


def test_idle_time_out_and_relaunch():
    """A loop that timed out while the host was busy is launched again by
    the next call, which still runs exactly one step."""
    n = 1500
    a, b = pair(n, 100, False)
    a.set_resident_step(20)
    plan = script(n, 60, 3)
    fa = []
    for t, (f, i) in enumerate(plan):
        fa.append(list(a.step(f, i)))
        if t % 4 == 1:
            time.sleep(0.002)  # 100 x the idle time
    fb = drive(b, plan, 0)
    assert fa == fb
    assert same_state(a, b, n)
    assert a.elapsed_simulation() == 60


def test_two_resident_simulations_alternate():
    """Two simulations with resident loops stepped in turn on one GPU: each
    loop waits for the other's idle time-out, and both stay exact."""
    n = 1200
    a, ref_a = pair(n, 100, True)
    b, ref_b = pair(n, 100, True)
    a.set_resident_step(50)
    b.set_resident_step(50)
    plan_a, plan_b = script(n, 80, 4), script(n, 80, 5)
    fa, fb = [], []
    for (f1, i1), (f2, i2) in zip(plan_a, plan_b):
        fa.append(list(a.step(f1, i1)))
        fb.append(list(b.step(f2, i2)))
    assert fa == drive(ref_a, plan_a, 0)
    assert fb == drive(ref_b, plan_b, 0)
    assert same_state(a, ref_a, n) and same_state(b, ref_b, n)


def test_switching_modes_mid_run():
    n = 2000
    a, b = pair(n)
    plan = script(n, 90, 6)
    fa = []
    for t, (f, i) in enumerate(plan):
        if t == 30:
            a.set_resident_step(0)
        if t == 60:
            a.set_resident_step(500)
        fa.append(list(a.step(f, i)))
    assert fa == drive(b, plan, 0)
    assert same_state(a, b, n)


def test_idle_time_limit_is_enforced():
    a, _ = pair(500, 50, False)
    with pytest.raises(nb.NemoError):
        a.set_resident_step(100001)
    a.set_resident_step(100000)
    assert len(a.step([1, 2, 3])) >= 3


def test_mixed_neuron_types_match_the_oracle():
    """IF_curr_exp, Izhikevich and Poisson neurons (Pareto out-degree,
    mixed-sign weights) stepped through the resident loop with firing and
    current stimuli: the same fired neurons as the oracle's step, and the
    same neuron state."""
    (np_, tp, idp) = nets.mixed_network(nb)
    (no_, to, ido) = nets.mixed_network(O)
    sim, ref = nb.Simulation(np_, nb.Configuration()), O.Simulation(no_, O.Configuration())
    n = len(idp[0]) + len(idp[1]) + 100
    rng = np.random.default_rng(8)
    fired = 0
    for t in range(300):
        f = rng.choice(n, 3, replace=False).tolist() if t % 4 == 0 else None
        i = [(int(a), float(v)) for a, v in zip(rng.choice(n, 5), rng.normal(0, 10, 5))] if t % 6 == 0 else None
        got = list(sim.step(f, i))
        assert got == list(ref.step(f, i)), t
        fired += len(got)
    assert fired > 100
    for t, ns, m in [(tp[0], 4, len(idp[0])), (tp[1], 2, len(idp[1]))]:
        a = np.asarray(sim.type_state(t, ns, m), np.float32)
        b = np.asarray(ref.type_state(t, ns, m), np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)) or np.array_equal(a, b, equal_nan=True)
