"""nemosim_b200 -- a B200 (sm_100a) simulation backend for the NeMo spiking
neural network simulator.

The native library (``lib/libnemo_b200.so``, C ABI in ``include/nemo_b200.h``)
is a drop-in for the reference C API (src/nemo.h).  This module binds it with
ctypes behind the interface of the reference's Python binding
(src/api/python/nemo_py.cpp:729-816 and src/api/python/__init__.py.in):
``Network``, ``Configuration`` and ``Simulation`` with the same method names,
argument meaning and errors (a ``NemoError`` carrying the reference status
code).  Vector arguments are accepted wherever the reference binding accepts
lists.
"""
from __future__ import annotations

import array

import ctypes as C

import numpy as np

from ._lib import lib, library_path  # noqa: F401

NEMO_OK = 0
NEMO_INVALID_INPUT = 6
NEMO_BACKEND_CUDA = 0
NEMO_BACKEND_CPU = 1


class NemoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check(code: int):
    if code != NEMO_OK:
        raise NemoError(code, lib().nemo_strerror().decode())


def _u32(x):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.uint32)))


def _f32(x):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float32)))


_EMPTY_U32 = np.zeros(1, np.uint32)
_EMPTY_F32 = np.zeros(1, np.float32)

# nemo_step bound with plain pointer arguments for Simulation.step, which is
# called once per simulated millisecond: the ndpointer checks of the general
# binding cost more than the call
_STEP_PROTO = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t,
                          C.c_void_p, C.c_void_p)
_step_fn = None


def _nemo_step():
    global _step_fn
    if _step_fn is None:
        _step_fn = _STEP_PROTO(("nemo_step", lib()))
    return _step_fn


def _u32_buffer(x):
    """x as a buffer of unsigned 32-bit ints (array.array for a list)."""
    return array.array("I", x) if isinstance(x, list) else _u32(x)


def _address(buf) -> int:
    return buf.buffer_info()[0] if isinstance(buf, array.array) else buf.ctypes.data


def add_plugin_path(directory: str):
    """nemo.add_plugin_path: a directory searched for neuron-type
    descriptors (<type>.ini) before ~/.nemo/plugins and the library's own
    plugins/ directory (src/nemo/NeuronType.cpp:45-70)."""
    _check(lib().nemo_add_plugin_path(str(directory).encode()))


def version() -> str:
    return lib().nemo_version().decode()


def cuda_device_count() -> int:
    n = C.c_uint()
    _check(lib().nemo_cuda_device_count(C.byref(n)))
    return n.value


class Configuration:
    """nemo::Configuration (src/nemo/Configuration.hpp)."""

    def __init__(self):
        self._h = lib().nemo_new_configuration()
        self._delete = lib().nemo_delete_configuration
        if not self._h:
            raise NemoError(10, lib().nemo_strerror().decode())

    def __del__(self):
        # the deleter was bound at construction (at interpreter exit this
        # module's globals may already be gone)
        if getattr(self, "_h", None):
            self._delete(self._h)
            self._h = None

    def set_stdp_function(self, prefire, postfire, *limits):
        """(pre, post, min_weight, max_weight) or (pre, post, minE, maxE, minI, maxI):
        the two overloads of Configuration::setStdpFunction
        (src/nemo/Configuration.cpp:80-100)."""
        if len(limits) == 2:
            min_w, max_w = limits
            limits = (0.0, max_w, 0.0, min_w)
        if len(limits) != 4:
            raise TypeError("set_stdp_function takes 2 or 4 weight limits")
        pre, post = _f32(prefire), _f32(postfire)
        _check(lib().nemo_set_stdp_function(self._h, pre, len(pre), post, len(post),
                                            *[float(v) for v in limits]))

    def set_cuda_backend(self, device: int = -1):
        _check(lib().nemo_set_cuda_backend(self._h, int(device)))

    def set_cpu_backend(self):
        _check(lib().nemo_set_cpu_backend(self._h))

    def set_write_only_synapses(self):
        _check(lib().nemo_set_write_only_synapses(self._h))

    def set_device_construction(self, on: bool = True):
        """Build the connectivity on the device where the network allows it
        (an extension; the default) or always on the host."""
        _check(lib().nemo_b200_set_device_construction(self._h, int(bool(on))))

    def backend_description(self) -> str:
        d = C.c_char_p()
        _check(lib().nemo_backend_description(self._h, C.byref(d)))
        return d.value.decode()


class Network:
    """nemo::Network (src/nemo/Network.hpp)."""

    def __init__(self, _handle=None):
        self._h = _handle if _handle is not None else lib().nemo_new_network()
        self._delete = lib().nemo_delete_network
        if not self._h:
            raise NemoError(10, lib().nemo_strerror().decode())

    def __del__(self):
        # the deleter was bound at construction (at interpreter exit this
        # module's globals may already be gone)
        if getattr(self, "_h", None):
            self._delete(self._h)
            self._h = None

    def add_neuron_type(self, name: str) -> int:
        t = C.c_uint()
        _check(lib().nemo_add_neuron_type(self._h, name.encode(), C.byref(t)))
        return t.value

    def add_neuron(self, ntype: int, idx, *args):
        """add_neuron(type, idx, p0, ..., s0, ...); idx and each argument may
        be a scalar or a vector (src/api/python/nemo_py.cpp add_neuron_va)."""
        idx = _u32(idx)
        n = len(idx)
        cols = [np.broadcast_to(_f32(a), (n,)) for a in args]
        mat = np.ascontiguousarray(np.stack(cols, axis=1), dtype=np.float32).reshape(-1) if cols else _EMPTY_F32
        _check(lib().nemo_b200_add_neurons(self._h, ntype, n, idx, len(args), mat))

    def add_synapse(self, source, target, delay, weight, plastic):
        """Returns the synapse id (or a vector of ids for vector arguments)."""
        src, tgt, dly = _u32(source), _u32(target), _u32(delay)
        w = _f32(weight)
        pl = np.ascontiguousarray(np.atleast_1d(np.asarray(plastic, dtype=np.uint8)))
        n = max(len(src), len(tgt), len(dly), len(w), len(pl))
        src, tgt, dly, w, pl = (np.ascontiguousarray(np.broadcast_to(a, (n,))) for a in (src, tgt, dly, w, pl))
        ids = np.zeros(max(n, 1), np.uint64)
        _check(lib().nemo_b200_add_synapses(self._h, n, src, tgt, dly, w, pl, ids))
        scalar = all(np.ndim(a) == 0 for a in (source, target, delay, weight, plastic))
        return int(ids[0]) if scalar else ids[:n]

    def neuron_count(self) -> int:
        c = C.c_uint()
        _check(lib().nemo_neuron_count(self._h, C.byref(c)))
        return c.value

    def _getf(self, fn, *args):
        v = C.c_float()
        _check(fn(self._h, *args, C.byref(v)))
        return v.value

    def get_neuron_state(self, idx, var):
        return self._getf(lib().nemo_get_neuron_state_n, idx, var)

    def get_neuron_parameter(self, idx, p):
        return self._getf(lib().nemo_get_neuron_parameter_n, idx, p)

    def set_neuron(self, idx, *args):
        a = _f32(args)
        _check(lib().nemo_set_neuron_n(self._h, idx, len(a), a))

    def set_neuron_state(self, idx, var, val):
        _check(lib().nemo_set_neuron_state_n(self._h, idx, var, float(val)))

    def set_neuron_parameter(self, idx, p, val):
        _check(lib().nemo_set_neuron_parameter_n(self._h, idx, p, float(val)))

    def get_synapses_from(self, source):
        p = C.POINTER(C.c_uint64)()
        n = C.c_size_t()
        _check(lib().nemo_get_synapses_from_n(self._h, source, C.byref(p), C.byref(n)))
        return [p[i] for i in range(n.value)]

    def _getu(self, fn, sid):
        v = C.c_uint()
        _check(fn(self._h, C.c_uint64(sid), C.byref(v)))
        return v.value

    def get_synapse_source(self, sid):
        return self._getu(lib().nemo_get_synapse_source_n, sid)

    def get_synapse_target(self, sid):
        return self._getu(lib().nemo_get_synapse_target_n, sid)

    def get_synapse_delay(self, sid):
        return self._getu(lib().nemo_get_synapse_delay_n, sid)

    def get_synapse_weight(self, sid):
        return self._getf(lib().nemo_get_synapse_weight_n, C.c_uint64(sid))

    def get_synapse_plastic(self, sid):
        v = C.c_ubyte()
        _check(lib().nemo_get_synapse_plastic_n(self._h, C.c_uint64(sid), C.byref(v)))
        return bool(v.value)


def scatter_probe(ops: int, elements: int, kind: int = 0, ctas: int = 0, device: int = 0, reps: int = 20) -> float:
    """Microseconds per launch of `ops` scattered operations into `elements`
    16-byte slots (kind 0: 64-bit reductions, 1: 32-bit reductions, 2:
    8-byte loads) -- the floor under the step's delivery (an extension)."""
    us = C.c_float()
    _check(lib().nemo_b200_scatter_probe(ops, elements, kind, ctas, device, reps, C.byref(us)))
    return us.value


def example_random(ncount: int, scount: int, dmax: int, stdp: bool, seed: int | None = None,
                   sigma_exc: float = 5.0, sigma_inh: float = 2.0) -> Network:
    """The reference's example network random::construct
    (src/examples/random.cpp:63-88); `seed` and the noise sigmas default to
    the reference's (5489, 5, 2)."""
    h = C.c_void_p()
    if seed is None and sigma_exc == 5.0 and sigma_inh == 2.0:
        _check(lib().nemo_b200_example_random(C.byref(h), ncount, scount, dmax, int(stdp)))
    else:
        _check(lib().nemo_b200_example_random_ex(C.byref(h), ncount, scount, dmax, int(stdp),
                                                 5489 if seed is None else seed, sigma_exc, sigma_inh))
    return Network(h.value)


class Simulation:
    """nemo::Simulation on the B200 backend."""

    def __init__(self, net: Network, conf: Configuration):
        h = lib().nemo_new_simulation(net._h, conf._h)
        if not h:
            raise NemoError(lib().nemo_b200_last_status(), lib().nemo_strerror().decode())
        self._h = h
        self._delete = lib().nemo_delete_simulation

    def __del__(self):
        # the deleter was bound at construction (at interpreter exit this
        # module's globals may already be gone)
        if getattr(self, "_h", None):
            self._delete(self._h)
            self._h = None

    def step(self, fstim=None, istim=None):
        """One 1 ms cycle; returns the fired neuron ids (src/api/python/__init__.py.in step)."""
        f = _u32_buffer(fstim) if fstim is not None and len(fstim) else None
        if istim:
            inid = _u32_buffer([p[0] for p in istim])
            icur = array.array("f", [p[1] for p in istim])
        else:
            inid = icur = None
        fired = C.c_void_p()
        n = C.c_size_t()
        _check(_nemo_step()(self._h, _address(f) if f is not None else None, 0 if f is None else len(f),
                            _address(inid) if inid is not None else None, _address(icur) if icur is not None else None,
                            0 if inid is None else len(inid), C.addressof(fired), C.addressof(n)))
        if n.value == 0:
            return []
        return array.array("I", C.string_at(fired.value, 4 * n.value)).tolist()

    def step_no_alloc(self, fstim=None, istim=None, capacity: int = 1 << 16):
        """step() through nemo_b200_step_no_alloc, which allocates nothing (an
        extension): returns (status code, fired ids).  Errors are status codes
        only (NEMO_INVALID_INPUT, NEMO_BUFFER_OVERFLOW, ...), not exceptions."""
        f = _u32(fstim) if fstim is not None and len(fstim) else _EMPTY_U32
        if istim:
            inid = _u32([p[0] for p in istim])
            icur = _f32([p[1] for p in istim])
        else:
            inid, icur = _EMPTY_U32, _EMPTY_F32
        out = np.zeros(max(capacity, 1), np.uint32)
        n = C.c_size_t()
        status = lib().nemo_b200_step_no_alloc(self._h, f, 0 if f is _EMPTY_U32 else len(f), inid, icur,
                                               0 if inid is _EMPTY_U32 else len(inid), out, capacity, C.byref(n))
        return status, out[:min(n.value, capacity)].tolist()

    def run(self, steps: int, stdp_period: int = 0, reward: float = 1.0, ids: bool = True,
            max_ids: int | None = None):
        """Device-resident run of `steps` unstimulated steps (an extension):
        returns (fired counts, synaptic events, fired ids or None)."""
        counts = np.zeros(max(steps, 1), np.uint32)
        events = np.zeros(max(steps, 1), np.uint64)
        cap = max_ids if max_ids is not None else steps * 4096
        buf = np.zeros(max(cap, 1), np.uint32) if ids else None
        ln = C.c_size_t()

        def ptr(a):
            return None if a is None else a.ctypes.data_as(C.c_void_p)
        _check(lib().nemo_b200_run(self._h, steps, stdp_period, reward, ptr(counts), ptr(events), ptr(buf),
                                   cap if buf is not None else 0, C.byref(ln)))
        if buf is None:
            return counts[:steps], events[:steps], None
        return counts[:steps], events[:steps], buf[: ln.value].copy()

    def apply_stdp(self, reward: float):
        _check(lib().nemo_apply_stdp(self._h, float(reward)))

    def _getf(self, fn, *args):
        v = C.c_float()
        _check(fn(self._h, *args, C.byref(v)))
        return v.value

    def get_neuron_state(self, idx, var):
        return self._getf(lib().nemo_get_neuron_state_s, idx, var)

    def get_neuron_parameter(self, idx, p):
        return self._getf(lib().nemo_get_neuron_parameter_s, idx, p)

    def get_membrane_potential(self, idx):
        return self._getf(lib().nemo_get_membrane_potential, idx)

    def set_neuron(self, idx, *args):
        a = _f32(args)
        _check(lib().nemo_set_neuron_s(self._h, idx, len(a), a))

    def set_neuron_state(self, idx, var, val):
        _check(lib().nemo_set_neuron_state_s(self._h, idx, var, float(val)))

    def set_neuron_parameter(self, idx, p, val):
        _check(lib().nemo_set_neuron_parameter_s(self._h, idx, p, float(val)))

    def get_synapses_from(self, source):
        p = C.POINTER(C.c_uint64)()
        n = C.c_size_t()
        _check(lib().nemo_get_synapses_from_s(self._h, source, C.byref(p), C.byref(n)))
        return [p[i] for i in range(n.value)]

    def _getu(self, fn, sid):
        v = C.c_uint()
        _check(fn(self._h, C.c_uint64(sid), C.byref(v)))
        return v.value

    def get_synapse_source(self, sid):
        return self._getu(lib().nemo_get_synapse_source_s, sid)

    def get_synapse_target(self, sid):
        return self._getu(lib().nemo_get_synapse_target_s, sid)

    def get_synapse_delay(self, sid):
        return self._getu(lib().nemo_get_synapse_delay_s, sid)

    def get_synapse_weight(self, sid):
        return self._getf(lib().nemo_get_synapse_weight_s, C.c_uint64(sid))

    def get_synapse_plastic(self, sid):
        v = C.c_ubyte()
        _check(lib().nemo_get_synapse_plastic_s(self._h, C.c_uint64(sid), C.byref(v)))
        return bool(v.value)

    def weights_fx(self, nsyn: int | None = None) -> np.ndarray:
        """All weights (raw Q11.20) in network iteration order (an extension)."""
        if nsyn is None:
            nsyn = self.synapse_count()
        out = np.zeros(max(nsyn, 1), np.int32)
        ln = C.c_size_t()
        _check(lib().nemo_b200_get_weights_fx(self._h, out, len(out), C.byref(ln)))
        return out[: ln.value]

    def type_state(self, ntype: int, nstate: int, n: int) -> np.ndarray:
        out = np.zeros(max(nstate * n, 1), np.float32)
        ln = C.c_size_t()
        _check(lib().nemo_b200_get_type_state(self._h, ntype, out, len(out), C.byref(ln)))
        return out[: ln.value].reshape(nstate, n) if ln.value else np.zeros((nstate, 0), np.float32)

    def synapse_count(self) -> int:
        v = C.c_uint64()
        _check(lib().nemo_b200_synapse_count(self._h, C.byref(v)))
        return v.value

    def set_profiling(self, on: bool = True):
        _check(lib().nemo_b200_set_profiling(self._h, int(on)))

    def set_graphs(self, on: bool = True):
        """CUDA-graph replay of run()'s step loop (an extension; on by default)."""
        _check(lib().nemo_b200_set_graphs(self._h, int(on)))

    def set_persistent(self, on: bool = True):
        """run()'s step loop as one persistent cooperative launch per segment
        between applyStdp calls (an extension; on by default) or as two
        launches per step."""
        _check(lib().nemo_b200_set_persistent(self._h, int(on)))

    def set_resident_step(self, idle_us: int = 200):
        """step() through a step loop that stays resident on the GPU between
        calls and ends after `idle_us` microseconds without one (an
        extension; 200 by default, 0 = two kernel launches per step)."""
        _check(lib().nemo_b200_set_resident_step(self._h, int(idle_us)))

    def trace_phases(self, steps: int = 100) -> np.ndarray:
        """Phase trace of one launch of the persistent loop (an extension):
        %globaltimer [steps, CTAs, 5] in ns."""
        cap = steps * 8192 * 5
        out = np.zeros(cap, np.uint64)
        ctas = C.c_uint()
        _check(lib().nemo_b200_trace_phases(self._h, steps, out, cap, C.byref(ctas)))
        return out[: steps * ctas.value * 5].reshape(steps, ctas.value, 5)

    def connectivity_digest(self):
        """(digests of the device connectivity and its delay-group count,
        built on the device) -- an extension; equal digests mean equal
        bytes."""
        out = np.zeros(10, np.uint64)
        _check(lib().nemo_b200_connectivity_digest(self._h, out))
        return [int(v) for v in out[:9]], bool(out[9])

    def set_wait_limit(self, polls: int):
        """Polls of each grid-barrier or request wait before it gives up and
        the call reports NEMO_CUDA_ERROR (an extension; 0: at once)."""
        _check(lib().nemo_b200_set_wait_limit(self._h, int(polls)))

    def run_stats(self) -> dict:
        """Statistics of the last run() (an extension): device ms, per-kernel
        ms and launches (when profiling; "step" and "stdp" are the update and
        deliver kernels of the two-launch step, "run" the persistent loop),
        spikes, events, STDP entries walked and the number of plastic
        synapses."""
        run_ms = C.c_float()
        kms = (C.c_float * 4)()
        kl = (C.c_uint * 4)()
        vals = [C.c_uint64() for _ in range(4)]
        _check(lib().nemo_b200_run_stats(self._h, C.byref(run_ms), kms, kl, *[C.byref(v) for v in vals]))
        names = ("step", "stdp", "apply", "run")
        return {"run_ms": run_ms.value,
                "kernel_ms": {n: kms[i] for i, n in enumerate(names)},
                "kernel_launches": {n: kl[i] for i, n in enumerate(names)},
                "fired": vals[0].value, "events": vals[1].value,
                "stdp_entries": vals[2].value, "plastic_synapses": vals[3].value}

    def set_launch(self, partition: int, threads: int):
        """Launch shape of the step kernel (an extension); results do not depend on it."""
        _check(lib().nemo_b200_set_launch(self._h, partition, threads))

    def launch(self):
        p, t = C.c_uint(), C.c_uint()
        _check(lib().nemo_b200_get_launch(self._h, C.byref(p), C.byref(t)))
        return p.value, t.value

    def autotune(self, trial_steps: int = 50) -> float:
        """Pick the fastest launch shape on trial steps run from a snapshot
        (the simulation state is restored); returns microseconds per step."""
        us = C.c_float()
        _check(lib().nemo_b200_autotune(self._h, trial_steps, C.byref(us)))
        return us.value

    def step_events(self) -> int:
        """Synaptic events of all step() calls so far (an extension)."""
        v = C.c_uint64()
        _check(lib().nemo_b200_step_events(self._h, C.byref(v)))
        return v.value

    def elapsed_wallclock(self):
        v = C.c_ulong()
        _check(lib().nemo_elapsed_wallclock(self._h, C.byref(v)))
        return v.value

    def elapsed_simulation(self):
        v = C.c_ulong()
        _check(lib().nemo_elapsed_simulation(self._h, C.byref(v)))
        return v.value

    def reset_timer(self):
        _check(lib().nemo_reset_timer(self._h))


class Batch(Simulation):
    """Independent networks advanced together (an extension).  run() returns
    fired counts as [step][network] and each step's fired ids network by
    network; every network's results equal its own Simulation's."""

    def __init__(self, networks, conf: Configuration):
        arr = (C.c_void_p * len(networks))(*[n._h for n in networks])
        h = lib().nemo_b200_new_batch(arr, len(networks), conf._h)
        if not h:
            raise NemoError(lib().nemo_b200_last_status(), lib().nemo_strerror().decode())
        self._h = h
        self._delete = lib().nemo_delete_simulation
        self.count = len(networks)

    def run(self, steps: int, stdp_period: int = 0, reward: float = 1.0, ids: bool = True,
            max_ids: int | None = None):
        counts = np.zeros(max(steps, 1) * self.count, np.uint32)
        events = np.zeros(max(steps, 1), np.uint64)
        cap = max_ids if max_ids is not None else steps * 65536
        buf = np.zeros(max(cap, 1), np.uint32) if ids else None
        ln = C.c_size_t()

        def ptr(a):
            return None if a is None else a.ctypes.data_as(C.c_void_p)
        _check(lib().nemo_b200_run(self._h, steps, stdp_period, reward, ptr(counts), ptr(events), ptr(buf),
                                   cap if buf is not None else 0, C.byref(ln)))
        counts = counts[: steps * self.count].reshape(steps, self.count)
        return counts, events[:steps], (buf[: ln.value].copy() if buf is not None else None)

    def streams(self, counts: np.ndarray, ids: np.ndarray):
        """Split a run's (counts, ids) into per-network (counts, ids)."""
        per_counts = [counts[:, k].copy() for k in range(self.count)]
        per_ids = [[] for _ in range(self.count)]
        pos = 0
        for t in range(counts.shape[0]):
            for k in range(self.count):
                c = int(counts[t, k])
                per_ids[k].append(ids[pos:pos + c])
                pos += c
        return [(per_counts[k], np.concatenate(per_ids[k]) if per_ids[k] else np.zeros(0, np.uint32))
                for k in range(self.count)]

    def type_state(self, net: int, ntype: int, nstate: int, n: int) -> np.ndarray:
        out = np.zeros(max(nstate * n, 1), np.float32)
        ln = C.c_size_t()
        _check(lib().nemo_b200_batch_get_type_state(self._h, net, ntype, out, len(out), C.byref(ln)))
        return out[: ln.value].reshape(nstate, n) if ln.value else np.zeros((nstate, 0), np.float32)


def host_nrand(state: np.ndarray) -> float:
    """Host build of the device's glibc-exact nrand (advances `state`)."""
    return lib().nemo_b200_host_nrand(state)


def libm_calibration():
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    _check(lib().nemo_b200_libm_calibration(C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


def libm_verify() -> int:
    """Arguments (of all 100,663,298 reachable ones) at which the host build
    of the device's logf/sinf differs from the host libm."""
    n = C.c_uint64()
    _check(lib().nemo_b200_libm_verify(C.byref(n)))
    return n.value
