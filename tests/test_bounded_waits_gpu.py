"""The bounded waits of the persistent and resident step loops.

Every wait of a CTA on the other CTAs -- the grid barriers of the persistent
step loop, the resident loop's request broadcast -- polls at most a set
number of times, then sets the loop's error word and ends the launch, so a
wait that cannot complete becomes an error status instead of a hung GPU.
These tests lower the limit to zero polls (nemo_b200_set_wait_limit), so
that the waits run out at once on a healthy GPU: nothing faults, traps or
hangs.  The call must return NEMO_CUDA_ERROR through the C ABI, the
simulation must delete cleanly, and a new simulation on the same device must
still run bit-exact against the oracle.
"""
import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

pytestmark = pytest.mark.gpu

NEMO_CUDA_ERROR = 4


def fresh_sim_is_bitexact():
    sp = nb.Simulation(nb.example_random(1000, 100, 20, True), nets.standard_stdp(nb))
    so = O.Simulation(O.example_random(1000, 100, 20, True), nets.standard_stdp(O))
    cp, _, ip = sp.run(300, 100, 1.0)
    co, io = so.run(300, 100, 1.0)
    assert cp.sum() > 0
    assert np.array_equal(cp, co) and np.array_equal(ip, io)
    # nemo_step through the resident loop as well
    assert [sp.step() for _ in range(50)] == [so.step() for _ in range(50)]
    assert np.array_equal(sp.weights_fx(100000), so.weights_fx(100000))


def test_grid_barrier_wait_runs_out():
    sim = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    assert sim.launch() is not None
    sim.set_wait_limit(0)
    with pytest.raises(nb.NemoError) as e:
        sim.run(100, 100, 1.0)
    assert e.value.code == NEMO_CUDA_ERROR
    assert "grid barrier" in str(e.value)
    del sim
    fresh_sim_is_bitexact()


def test_resident_request_wait_runs_out():
    sim = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    sim.set_wait_limit(0)
    with pytest.raises(nb.NemoError) as e:
        for _ in range(10):
            sim.step([1])
    assert e.value.code == NEMO_CUDA_ERROR
    del sim
    fresh_sim_is_bitexact()


def test_default_limit_does_not_run_out():
    """The default limit (seconds of polling) never runs out on a working
    step, and setting it explicitly changes no result."""
    a = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b = nb.Simulation(nb.example_random(3000, 150, 20, True), nets.standard_stdp(nb))
    b.set_wait_limit(1 << 24)
    ra = a.run(300, 100, 1.0)
    rb = b.run(300, 100, 1.0)
    assert np.array_equal(ra[2], rb[2])
    assert [a.step() for _ in range(20)] == [b.step() for _ in range(20)]
