"""nemo_b200_step_no_alloc (the allocation-free nemo_step) against nemo_step:
two stimulated steps in a row give the same fired neurons and leave the
same simulation state, and its size, index and capacity errors leave the
simulation as it was (or, for the fired-list capacity, step exactly as
nemo_step does).  This file is collected last and needs no other test."""
import ctypes

import numpy as np
import pytest

import nemosim_b200 as nb
from tests import nets

pytestmark = pytest.mark.gpu

NEMO_OK, NEMO_INVALID_INPUT, NEMO_BUFFER_OVERFLOW = 0, 6, 7
STIMULUS_MAX = 65536


def twins():
    make = lambda: nb.Simulation(nb.example_random(1000, 100, 20, True), nets.standard_stdp(nb))
    return make(), make()


def same_state(a, b):
    sa, sb = a.type_state(0, 2, 1000), b.type_state(0, 2, 1000)
    return np.array_equal(np.asarray(sa, np.float32).view(np.uint32), np.asarray(sb, np.float32).view(np.uint32))


STIMULI = [
    # firing stimulus, current stimulus (neuron 5 twice: the last value wins)
    ([3, 17, 500], [(5, 10.0), (700, -3.0), (5, 12.5), (42, 7.0)]),
    ([999, 0], [(17, 25.0), (17, 0.5)]),
]


def test_two_steps_match_nemo_step():
    ref, sim = twins()
    for fstim, istim in STIMULI:
        expected = ref.step(fstim, istim)
        status, fired = sim.step_no_alloc(fstim, istim)
        assert status == NEMO_OK
        assert fired == expected
        assert 3 in fired or fstim != STIMULI[0][0]
    assert same_state(ref, sim)
    # the rest of the simulation (pending deliveries, STDP) is identical too
    a = ref.run(200, 100, 1.0)
    b = sim.run(200, 100, 1.0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[2], b[2])
    assert np.array_equal(ref.weights_fx(100000), sim.weights_fx(100000))


def test_oversize_stimulus_is_rejected_without_stepping():
    ref, sim = twins()
    status, fired = sim.step_no_alloc([0] * (STIMULUS_MAX + 1))
    assert status == NEMO_BUFFER_OVERFLOW and fired == []
    status, _ = sim.step_no_alloc([1] * 10, [(2, 1.0)] * (STIMULUS_MAX // 2))
    assert status == NEMO_BUFFER_OVERFLOW
    assert sim.elapsed_simulation() == 0
    # the largest stimulus that fits is accepted
    status, fired = sim.step_no_alloc([7] * (STIMULUS_MAX - 2), [(8, 1.0)])
    assert status == NEMO_OK and 7 in fired
    assert ref.step([7], [(8, 1.0)]) == fired
    assert same_state(ref, sim)


def test_invalid_index_is_rejected_without_stepping():
    ref, sim = twins()
    assert sim.step_no_alloc([10 ** 7])[0] == NEMO_INVALID_INPUT
    assert sim.step_no_alloc([1], [(10 ** 7, 1.0)])[0] == NEMO_INVALID_INPUT
    assert sim.elapsed_simulation() == 0
    assert sim.step_no_alloc([4])[1] == ref.step([4])
    assert same_state(ref, sim)


def test_small_fired_capacity_reports_overflow_after_stepping():
    ref, sim = twins()
    expected = ref.step([3, 4, 5])
    status, fired = sim.step_no_alloc([3, 4, 5], capacity=1)
    assert status == NEMO_BUFFER_OVERFLOW
    assert fired == expected[:1]
    assert sim.elapsed_simulation() == 1
    assert same_state(ref, sim)


class _MallInfo2(ctypes.Structure):
    _fields_ = [(name, ctypes.c_size_t) for name in
                ("arena", "ordblks", "smblks", "hblks", "hblkhd", "usmblks", "fsmblks", "uordblks", "fordblks",
                 "keepcost")]


def test_call_allocates_nothing():
    """The entry point's defining property, measured: after a warm-up call
    (which looks up the static buffer's device address and loads the
    stimulus kernel), a stimulated call leaves the device's free memory
    (cudaMemGetInfo) and the host heap in use (glibc mallinfo2, all arenas)
    exactly as they were.  The call is made through a plain C function
    pointer with every argument prepared beforehand, and Python's garbage
    collector is paused, so that nothing but the call itself runs between
    the two readings."""
    import gc

    import torch

    libc = ctypes.CDLL("libc.so.6")
    libc.mallinfo2.restype = _MallInfo2
    step = ctypes.CDLL(nb.library_path()).nemo_b200_step_no_alloc
    step.restype = ctypes.c_int
    step.argtypes = [ctypes.c_void_p] * 9
    _, sim = twins()
    fstim = np.array([3, 17, 500], np.uint32)
    inidx = np.array([5, 700, 5], np.uint32)
    icur = np.array([10.0, -3.0, 12.5], np.float32)
    fired = np.zeros(1 << 16, np.uint32)
    nfired = ctypes.c_size_t()
    args = (ctypes.c_void_p(sim._h), ctypes.c_void_p(fstim.ctypes.data), ctypes.c_void_p(len(fstim)),
            ctypes.c_void_p(inidx.ctypes.data), ctypes.c_void_p(icur.ctypes.data), ctypes.c_void_p(len(inidx)),
            ctypes.c_void_p(fired.ctypes.data), ctypes.c_void_p(len(fired)),
            ctypes.c_void_p(ctypes.addressof(nfired)))
    assert step(*args) == NEMO_OK  # warm-up
    assert step(*args) == NEMO_OK
    torch.cuda.mem_get_info(0)
    gc.disable()
    try:
        free0 = torch.cuda.mem_get_info(0)[0]
        rc_device = step(*args)
        free1 = torch.cuda.mem_get_info(0)[0]
        heap0 = libc.mallinfo2().uordblks
        rc_host = step(*args)
        heap1 = libc.mallinfo2().uordblks
    finally:
        gc.enable()
    assert rc_device == NEMO_OK and rc_host == NEMO_OK
    assert free1 == free0, f"device free memory changed by {free1 - free0} bytes"
    assert heap1 == heap0, f"host heap in use changed by {heap1 - heap0} bytes"
    assert 3 in fired[:nfired.value]
