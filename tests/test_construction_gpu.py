"""The connectivity built on the device against the host build.

Every case builds the same network twice -- once with the device build (the
default) and once with it turned off -- and checks that the device memory
holds the same bytes (digests of the forward matrix, its row starts, the
delay-group ends and masks, and the reverse matrix of plastic synapses),
that the two simulations fire the same spikes and reach the same weights,
and that the synapse queries answer alike.  The errors of a bad network
(a synapse to a missing neuron, a weight outside the fixed-point range)
are the host build's, in the same order.  The host build is the one the
oracle parity tests pinned first; the full-size parity tests run the
device build against the oracle directly.
"""
import gc
import time

import numpy as np
import pytest

import nemosim_b200 as nb
from tests import nets

pytestmark = pytest.mark.gpu

f32 = np.float32


def build(make_net, make_conf, device):
    conf = make_conf()
    conf.set_device_construction(device)
    return nb.Simulation(make_net(), conf)


def both(make_net, make_conf=nb.Configuration, expect_device=True):
    """(device-built, host-built) simulations of the same network, with
    equal digests."""
    sd = build(make_net, make_conf, True)
    sh = build(make_net, make_conf, False)
    dd, on_dev = sd.connectivity_digest()
    dh, on_host = sh.connectivity_digest()
    assert on_dev == expect_device
    assert not on_host
    assert dd == dh
    return sd, sh


def same_run(sd, sh, ms=300, period=100):
    cd, ed, idd = sd.run(ms, period, 1.0)
    ch, eh, idh = sh.run(ms, period, 1.0)
    assert np.array_equal(cd, ch)
    assert np.array_equal(ed, eh)
    assert np.array_equal(idd, idh)
    assert cd.sum() > 0
    return int(cd.sum())


def same_queries(sd, sh, sources):
    for s in sources:
        ids = list(sd.get_synapses_from(int(s)))
        assert ids == list(sh.get_synapses_from(int(s)))
        for i in ids:
            for q in ("get_synapse_target", "get_synapse_delay", "get_synapse_weight", "get_synapse_plastic"):
                assert getattr(sd, q)(i) == getattr(sh, q)(i), (q, i)


def test_random_stdp_network():
    sd, sh = both(lambda: nb.example_random(3000, 150, 20, True), lambda: nets.standard_stdp(nb))
    same_queries(sd, sh, range(0, 3000, 97))
    same_run(sd, sh, 500, 100)
    assert np.array_equal(sd.weights_fx(3000 * 150), sh.weights_fx(3000 * 150))
    same_queries(sd, sh, range(5, 3000, 211))


def test_offset_ring_and_queries_before_and_after_a_run():
    def make():
        return nets.create_ring(nb, nb.Network(), 1500, 1_000_000)

    sd, sh = both(make)
    ring = np.arange(1_000_000, 1_001_500)
    same_queries(sd, sh, ring[::50])
    for s in (sd, sh):
        s.step(fstim=[1_000_000])
    same_run(sd, sh, 200, 0)


def test_sparse_ids_fall_back_to_the_host_build():
    def make():
        net = nb.Network()
        iz = net.add_neuron_type("Izhikevich")
        ids = (np.arange(2000, dtype=np.uint32) * 4099) + 17
        net.add_neuron(iz, ids, *nets.exc_neuron_args(5.0))
        rng = np.random.default_rng(3)
        src = np.repeat(ids, 40)
        tgt = rng.choice(ids, src.size).astype(np.uint32)
        net.add_synapse(src, tgt, rng.integers(1, 21, src.size).astype(np.uint32),
                        rng.uniform(0, 8, src.size).astype(f32), np.ones(src.size, np.uint8))
        return net

    sd, sh = both(make, lambda: nets.standard_stdp(nb), expect_device=False)
    same_run(sd, sh, 200, 100)


def test_mixed_types_interleaved_ids():
    sd, sh = both(lambda: nets.mixed_network(nb)[0], lambda: nets.standard_stdp(nb))
    same_run(sd, sh, 300, 100)


def test_row_longer_than_65535_uses_the_wide_group_table():
    def make():
        net = nb.Network()
        iz = net.add_neuron_type("Izhikevich")
        n = 1000
        net.add_neuron(iz, np.arange(n, dtype=np.uint32), *nets.exc_neuron_args(5.0))
        rng = np.random.default_rng(9)
        src = np.concatenate([np.zeros(70_000, np.uint32), np.repeat(np.arange(1, n, dtype=np.uint32), 20)])
        tgt = rng.integers(0, n, src.size).astype(np.uint32)
        dly = rng.integers(1, 11, src.size).astype(np.uint32)
        w = rng.uniform(0, 0.5, src.size).astype(f32)
        net.add_synapse(src, tgt, dly, w, np.ones(src.size, np.uint8))
        return net

    sd, sh = both(make, lambda: nets.standard_stdp(nb))
    same_run(sd, sh, 200, 100)
    same_queries(sd, sh, [0, 1, 999])


@pytest.mark.parametrize("dmax", [1, 63, 64])
def test_delay_extremes(dmax):
    def make():
        net = nb.Network()
        iz = net.add_neuron_type("Izhikevich")
        n = 500
        net.add_neuron(iz, np.arange(n, dtype=np.uint32), *nets.exc_neuron_args(5.0))
        rng = np.random.default_rng(dmax)
        src = np.repeat(np.arange(n, dtype=np.uint32), 30)
        tgt = rng.integers(0, n, src.size).astype(np.uint32)
        dly = rng.integers(1, dmax + 1, src.size).astype(np.uint32)
        dly[0] = dmax
        net.add_synapse(src, tgt, dly, rng.uniform(0, 6, src.size).astype(f32), np.ones(src.size, np.uint8))
        return net

    conf = (lambda: nets.standard_stdp(nb, n=20)) if dmax <= 44 else nb.Configuration
    sd, sh = both(make, conf)
    same_run(sd, sh, 200, 100 if dmax <= 44 else 0)


def test_no_synapses_and_no_plastic_synapses():
    def empty():
        net = nb.Network()
        iz = net.add_neuron_type("Izhikevich")
        net.add_neuron(iz, np.arange(64, dtype=np.uint32), *nets.exc_neuron_args(5.0))
        return net

    sd, sh = both(empty, lambda: nets.standard_stdp(nb))
    same_run(sd, sh, 100, 50)
    sd, sh = both(lambda: nb.example_random(500, 40, 10, False), lambda: nets.standard_stdp(nb))
    same_run(sd, sh, 200, 100)


def test_write_only_synapses():
    def conf():
        c = nb.Configuration()
        c.set_write_only_synapses()
        return c

    sd, sh = both(lambda: nb.example_random(800, 60, 20, False), conf)
    for s in (sd, sh):
        with pytest.raises(nb.NemoError) as e:
            s.get_synapses_from(0)
        assert e.value.code == nb.NEMO_INVALID_INPUT
    same_run(sd, sh, 200, 0)


def bad_network(bad_tgt_at=None, bad_src_at=None, bad_w_at=None):
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    net.add_neuron(iz, np.arange(100, dtype=np.uint32), *nets.exc_neuron_args(5.0))
    src = np.arange(100, dtype=np.uint32)
    tgt = (src + 1) % 100
    w = np.full(100, 1.0, f32)
    if bad_tgt_at is not None:
        tgt[bad_tgt_at] = 5000
    if bad_src_at is not None:
        src[bad_src_at] = 100
    if bad_w_at is not None:
        w[bad_w_at] = 3.0e3
    net.add_synapse(src, tgt, np.ones(100, np.uint32), w, np.zeros(100, np.uint8))
    return net


@pytest.mark.parametrize("bad", [dict(bad_tgt_at=7), dict(bad_src_at=9), dict(bad_w_at=4),
                                 dict(bad_tgt_at=7, bad_w_at=4), dict(bad_w_at=8, bad_src_at=8),
                                 dict(bad_src_at=20, bad_tgt_at=20)])
def test_errors_match_the_host_build(bad):
    got = []
    for device in (True, False):
        conf = nb.Configuration()
        conf.set_device_construction(device)
        with pytest.raises(nb.NemoError) as e:
            nb.Simulation(bad_network(**bad), conf)
        got.append((e.value.code, str(e.value)))
    assert got[0] == got[1]


def test_c2_network_digests_and_build_time():
    """The 100,000 x 1000 random network with STDP: the same bytes both
    ways; the device build's wall time is printed beside the host build's."""
    net = nb.example_random(100_000, 1000, 20, True)
    out = {}
    for device in (True, False):
        conf = nets.standard_stdp(nb)
        conf.set_device_construction(device)
        t0 = time.perf_counter()
        sim = nb.Simulation(net, conf)
        dt = time.perf_counter() - t0
        out[device] = (sim.connectivity_digest(), dt)
        if device:
            counts, _, _ = sim.run(100, 100, 1.0, ids=False)
            assert counts.sum() > 0
        del sim
        gc.collect()
    (dd, on_dev), t_dev = out[True]
    (dh, on_host), t_host = out[False]
    print(f"C2 construction: device {t_dev:.2f} s, host {t_host:.2f} s")
    assert on_dev and not on_host
    assert dd == dh


def batch_specs(seed, count, stdp):
    rng = np.random.default_rng(seed)
    return [dict(ncount=int(rng.integers(300, 2500)), scount=int(rng.integers(20, 200)), seed=100 + 7 * k,
                 sigma=float(rng.uniform(2, 8)), stdp=stdp) for k in range(count)]


def batch_net(s):
    return nb.example_random(s["ncount"], s["scount"], 20, s["stdp"], seed=s["seed"],
                             sigma_exc=s["sigma"], sigma_inh=s["sigma"])


def both_batch(specs, make_conf, expect_device=True, extra=None):
    out = []
    for device in (True, False):
        conf = make_conf()
        conf.set_device_construction(device)
        networks = [batch_net(s) for s in specs] + ([extra()] if extra else [])
        out.append(nb.Batch(networks, conf))
    (dd, on_dev), (dh, on_host) = out[0].connectivity_digest(), out[1].connectivity_digest()
    assert on_dev == expect_device and not on_host
    assert dd == dh
    return out


@pytest.mark.parametrize("stdp", [False, True])
def test_batch_of_one_type_networks(stdp):
    """A batch whose networks have one neuron type each is built on the
    device network by network, into the same union arrays."""
    bd, bh = both_batch(batch_specs(4, 7, stdp), (lambda: nets.standard_stdp(nb)) if stdp else nb.Configuration)
    cd, _, idd = bd.run(300, 100 if stdp else 0, 1.0)
    ch, _, idh = bh.run(300, 100 if stdp else 0, 1.0)
    assert np.array_equal(cd, ch) and np.array_equal(idd, idh)
    assert cd.sum() > 0


def test_batch_with_a_mixed_type_network_falls_back():
    bd, bh = both_batch(batch_specs(5, 3, False), nb.Configuration, expect_device=False,
                        extra=lambda: nets.mixed_network(nb, n_if=200, n_iz=300, n_poisson=50, seed=1)[0])
    cd, _, idd = bd.run(200)
    ch, _, idh = bh.run(200)
    assert np.array_equal(cd, ch) and np.array_equal(idd, idh)


def test_batch_error_names_the_first_bad_synapse():
    got = []
    for device in (True, False):
        conf = nb.Configuration()
        conf.set_device_construction(device)
        networks = [batch_net(s) for s in batch_specs(6, 3, False)] + [bad_network(bad_tgt_at=11, bad_w_at=30)]
        with pytest.raises(nb.NemoError) as e:
            nb.Batch(networks, conf)
        got.append((e.value.code, str(e.value)))
    assert got[0] == got[1]


def test_failed_construction_frees_device_memory():
    """A simulation whose construction fails (here at its last synapse,
    after the device arrays were allocated) frees them: five failed
    attempts at a 20M-synapse network leave the free device memory as it
    was."""
    import torch

    def attempt():
        net = nb.example_random(20_000, 1000, 20, True)
        net.add_synapse(0, 1_000_000, 1, 1.0, False)
        with pytest.raises(nb.NemoError) as e:
            nb.Simulation(net, nets.standard_stdp(nb))
        assert e.value.code == nb.NEMO_INVALID_INPUT

    attempt()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(5):
        attempt()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free0 - free1 < (64 << 20), (free0, free1)
