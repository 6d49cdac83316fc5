"""CPU tests of the C ABI: the library loads, exports every function that
include/nemo_b200.h declares, and its host-side logic (network construction,
queries, errors, the libm calibration) behaves like the reference."""
import ctypes
import os
import re

import numpy as np
import pytest

import nemosim_b200 as nb
import oracle as O
from tests import nets

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "nemo_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
    return sorted(set(re.findall(r"NEMO_B200_API\s+[^;(]*?\b(\w+)\s*\(", text)))


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(nb.library_path())
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from nemosim_b200._lib import SIGNATURES
    assert set(names) == set(SIGNATURES), set(names) ^ set(SIGNATURES)


def test_library_loaded_from_tree():
    path = nb.library_path()
    assert os.path.exists(path)
    assert path.startswith(os.path.join(ROOT, "nemosim_b200"))
    nb.lib()
    maps = open("/proc/self/maps").read()
    assert path in maps


def test_libm_calibration_is_exact():
    """The device's glibc-exact nrand, built for the host, equals the host
    libm nrand of the oracle (src/nemo/RNG.cpp:25-33) on random states."""
    log_flips, sin_flips, exc = nb.libm_calibration()
    assert exc == 0
    assert 0 < log_flips < (1 << 24) and 0 < sin_flips < 83886081
    rng = np.random.default_rng(11)
    for _ in range(20000):
        s = rng.integers(0, 2**32, 4, dtype=np.uint64).astype(np.uint32)
        s2 = s.copy()
        a, b = nb.host_nrand(s), O.nrand(s2)
        assert np.float32(a).tobytes() == np.float32(b).tobytes() or (a != a and b != b)
        assert np.array_equal(s, s2)


def test_libm_emulation_is_exact_at_every_argument():
    """logf over all 2^24 + 1 values of 1 - b and sinf over all 83,886,081
    values of a that nrand can produce (src/nemo/RNG.cpp:27-32): the host
    build of the device functions, with the flip table read only near float
    rounding midpoints, returns the libm's bits everywhere."""
    assert nb.libm_verify() == 0


def _state_for(u1: int, u2: int) -> np.ndarray:
    """A xorshift128 state whose next two draws are u1 and u2
    (src/nemo/RNG.cpp:9-18): with s0 = 0 the first draw is s3 ^ (s3 >> 19),
    and s1 sets the second through t = s1 ^ (s1 << 11)."""
    M = 0xffffffff

    def f(w):
        return (w ^ (w >> 19)) & M
    s3 = (u1 ^ (u1 >> 19)) & M           # inverse of f on 32 bits
    y = (f(u1) ^ u2) & M                 # needed t ^ (t >> 8)
    t = (y ^ (y >> 8) ^ (y >> 16) ^ (y >> 24)) & M
    s1 = (t ^ (t << 11) ^ (t << 22)) & M
    st = np.array([0, s1, 0, s3], np.uint32)
    chk = st.copy()
    assert O.urand(chk) == u1 and O.urand(chk) == u2
    return st


def test_libm_edge_arguments():
    """Draws at the ends of the argument ranges: u = 0, float(u) rounding to
    2^32 (then 1 - b == 0 and logf = -inf), and the 2^24 boundary."""
    edges = (0, 1, 127, 128, 2**24 - 1, 2**24, 2**24 + 1, 2**31, 2**32 - 129, 2**32 - 128, 2**32 - 1)
    for u1 in edges:
        for u2 in edges:
            a = _state_for(u1, u2)
            b = a.copy()
            x, y = nb.host_nrand(a), O.nrand(b)
            assert np.float32(x).tobytes() == np.float32(y).tobytes() or (x != x and y != y), (u1, u2, x, y)


def test_network_construction_and_queries():
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    assert net.add_neuron_type("Izhikevich") == iz
    net.add_neuron(iz, [3, 7, 9], *nets.exc_neuron_args(5.0))
    assert net.neuron_count() == 3
    sid = net.add_synapse(3, 7, 4, 0.25, True)
    assert sid == (3 << 32)
    ids = net.add_synapse([3, 3], [9, 7], [1, 2], [0.5, -0.5], [0, 1])
    assert list(ids) == [(3 << 32) | 1, (3 << 32) | 2]
    assert net.get_synapses_from(3) == [(3 << 32) | i for i in range(3)]
    assert net.get_synapse_target((3 << 32) | 1) == 9
    assert net.get_synapse_delay((3 << 32) | 2) == 2
    assert net.get_synapse_weight((3 << 32) | 2) == -0.5
    assert net.get_synapse_plastic((3 << 32) | 0)
    assert net.get_neuron_parameter(7, 4) == 5.0
    net.set_neuron_state(7, 1, -70.0)
    assert net.get_neuron_state(7, 1) == -70.0
    with pytest.raises(nb.NemoError) as e:
        net.get_neuron_state(8, 0)
    assert e.value.code == 6
    with pytest.raises(nb.NemoError):
        net.add_synapse(3, 7, 0, 1.0, False)  # delay 0 (NetworkImpl.cpp:115-118)
    with pytest.raises(nb.NemoError) as e:
        net.add_neuron(iz, 3, *nets.exc_neuron_args())  # duplicate index
    assert e.value.code == 6
    with pytest.raises(nb.NemoError):
        net.add_neuron(iz, 100, 1.0, 2.0)  # wrong argument count
    with pytest.raises(nb.NemoError):
        net.add_neuron_type("NoSuchType")


def test_stdp_configuration_errors():
    """testInvalidBounds / testInvalidStaticLength (src/test/stdp.cpp:291-338)"""
    pre = [np.exp(-dt / 20.0) for dt in range(20)]
    for lim in [(-0.01, 1.0, -0.01, -1.0), (0.01, -1.0, -0.01, -1.0), (-0.01, -1.0, -0.01, -1.0),
                (0.01, 1.0, 0.01, -1.0), (0.01, 1.0, -0.01, 1.0), (0.01, 1.0, 0.01, 1.0),
                (1.0, 0.01, -0.01, -1.0), (0.01, 1.0, -1.0, -0.01)]:
        for mod in (nb, O):
            with pytest.raises(mod.NemoError):
                mod.Configuration().set_stdp_function(pre, pre, *lim)
    long = [np.exp(-dt / 35.0) for dt in range(35)]
    for mod in (nb, O):
        with pytest.raises(mod.NemoError):
            mod.Configuration().set_stdp_function(long, long, 0.01, 1.0, -0.01, -1.0)


def test_example_generator_matches_oracle():
    """The native random::construct equals the oracle's restatement."""
    a = nb.example_random(300, 40, 20, True)
    b = O.example_random(300, 40, 20, True)
    sb = b.synapses()
    for i, sid in enumerate([(n << 32) | k for n in range(300) for k in range(40)][:2000]):
        assert a.get_synapse_target(sid) == sb[1][i]
        assert a.get_synapse_delay(sid) == sb[2][i]
        assert np.float32(a.get_synapse_weight(sid)) == sb[3][i]
        assert a.get_synapse_plastic(sid) == bool(sb[4][i])
    assert a.neuron_count() == 300
    ob = O.Simulation(b, O.Configuration())
    for n in (0, 239, 240, 299):
        for p in range(5):
            assert np.float32(a.get_neuron_parameter(n, p)) == np.float32(ob.get_neuron_parameter(n, p))
        for v in range(2):
            assert np.float32(a.get_neuron_state(n, v)) == np.float32(ob.get_neuron_state(n, v))


def test_set_neuron_on_the_network():
    """testSetNeuron's network half (src/test/test.cpp:769-835) on the
    product's host-side network"""
    from tests import kat
    kat.set_neuron_network(nb)
