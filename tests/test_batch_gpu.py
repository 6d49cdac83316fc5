"""The batched mode: independent networks advanced together in one launch
per step.  Each network's fire stream and state must equal its own
single-network run (and hence the oracle's)."""
import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

pytestmark = pytest.mark.gpu


def sweep(seed=0, count=6, lo=300, hi=2000, flo=30, fhi=150, dmax=20, stdp=False):
    """Networks of uneven size and fan-out, each with its own generator seed
    and input-noise sigma drawn from U(2, 8) (the batched configuration,
    scaled down)."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(count):
        specs.append(dict(ncount=int(rng.integers(lo, hi + 1)), scount=int(rng.integers(flo, fhi + 1)),
                          dmax=dmax, stdp=stdp, seed=1000 + 17 * k, sigma=float(rng.uniform(2, 8))))
    return specs


def build(mod, s):
    return mod.example_random(s["ncount"], s["scount"], s["dmax"], s["stdp"], seed=s["seed"],
                              sigma_exc=s["sigma"], sigma_inh=s["sigma"])


def test_batch_equals_individual_runs():
    specs = sweep()
    batch = nb.Batch([build(nb, s) for s in specs], nb.Configuration())
    counts, _, ids = batch.run(400)
    streams = batch.streams(counts, ids)
    for s, (c, i) in zip(specs, streams):
        sim = nb.Simulation(build(nb, s), nb.Configuration())
        c1, _, i1 = sim.run(400)
        assert c1.sum() > 0
        assert np.array_equal(c, c1) and np.array_equal(i, i1)
    for k, s in enumerate(specs):
        sim = nb.Simulation(build(nb, s), nb.Configuration())
        sim.run(400, ids=False)
        a = batch.type_state(k, 0, 2, s["ncount"])
        b = sim.type_state(0, 2, s["ncount"])
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_batch_member_matches_oracle():
    s = sweep(seed=3, count=3)[1]
    batch = nb.Batch([build(nb, x) for x in sweep(seed=3, count=3)], nb.Configuration())
    counts, _, ids = batch.run(300)
    c, i = batch.streams(counts, ids)[1]
    so = O.Simulation(build(O, s), O.Configuration())
    co, io = so.run(300)
    assert np.array_equal(c, co) and np.array_equal(i, io)


@pytest.mark.parametrize("persistent", [True, False])
def test_batch_with_stdp_and_launch_shapes(persistent):
    specs = sweep(seed=5, count=4, stdp=True)
    batch = nb.Batch([build(nb, s) for s in specs], nets.standard_stdp(nb))
    batch.set_persistent(persistent)
    batch.set_launch(64, 64)
    counts, _, ids = batch.run(300, 100, 1.0)
    streams = batch.streams(counts, ids)
    for s, (c, i) in zip(specs, streams):
        sim = nb.Simulation(build(nb, s), nets.standard_stdp(nb))
        c1, _, i1 = sim.run(300, 100, 1.0)
        assert np.array_equal(c, c1) and np.array_equal(i, i1)


def test_batch_mixed_types_in_different_orders():
    """Networks whose neuron types were added in different orders."""
    (a, _, _) = nets.mixed_network(nb, n_if=200, n_iz=300, n_poisson=50, seed=1)
    (b, _, _) = nets.mixed_network(nb, n_if=150, n_iz=100, n_poisson=80, seed=2)
    net_c = nb.Network()
    ps = net_c.add_neuron_type("PoissonSource")
    iz = net_c.add_neuron_type("Izhikevich")
    net_c.add_neuron(ps, np.arange(100, 160, dtype=np.uint32), 0.02)
    net_c.add_neuron(iz, np.arange(0, 100, dtype=np.uint32), *nets.exc_neuron_args(3.0))
    net_c.add_synapse(np.arange(100, 160, dtype=np.uint32), np.arange(0, 60, dtype=np.uint32), 3, 4.0, False)
    batch = nb.Batch([a, b, net_c], nb.Configuration())
    counts, _, ids = batch.run(300)
    streams = batch.streams(counts, ids)
    singles = [nets.mixed_network(nb, n_if=200, n_iz=300, n_poisson=50, seed=1)[0],
               nets.mixed_network(nb, n_if=150, n_iz=100, n_poisson=80, seed=2)[0]]
    net_c2 = nb.Network()
    ps = net_c2.add_neuron_type("PoissonSource")
    iz = net_c2.add_neuron_type("Izhikevich")
    net_c2.add_neuron(ps, np.arange(100, 160, dtype=np.uint32), 0.02)
    net_c2.add_neuron(iz, np.arange(0, 100, dtype=np.uint32), *nets.exc_neuron_args(3.0))
    net_c2.add_synapse(np.arange(100, 160, dtype=np.uint32), np.arange(0, 60, dtype=np.uint32), 3, 4.0, False)
    singles.append(net_c2)
    for net, (c, i) in zip(singles, streams):
        c1, _, i1 = nb.Simulation(net, nb.Configuration()).run(300)
        assert np.array_equal(c, c1) and np.array_equal(i, i1)


def test_batch_autotune_keeps_results():
    specs = sweep(seed=9, count=5)
    b1 = nb.Batch([build(nb, s) for s in specs], nb.Configuration())
    b2 = nb.Batch([build(nb, s) for s in specs], nb.Configuration())
    b2.run(50, ids=False)
    b1.run(50, ids=False)
    b2.autotune(10)
    r1 = b1.run(200)
    r2 = b2.run(200)
    assert np.array_equal(r1[0], r2[0]) and np.array_equal(r1[2], r2[2])
