"""ctypes wrapper of the oracle library (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libnemo_oracle.so")
_lock = threading.Lock()
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc, -O2 -ffp-contract=off)."""
    src = os.path.join(_HERE, "nemo_oracle.c")
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


class NemoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(_SO)
            vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
            sig = {
                "nemo_oracle_strerror": (C.c_char_p, []),
                "nemo_oracle_new_configuration": (vp, []),
                "nemo_oracle_delete_configuration": (None, [vp]),
                "nemo_oracle_set_stdp_function": (i, [vp, f32p, sz, f32p, sz, C.c_float, C.c_float, C.c_float, C.c_float]),
                "nemo_oracle_set_write_only_synapses": (i, [vp]),
                "nemo_oracle_new_network": (vp, []),
                "nemo_oracle_delete_network": (None, [vp]),
                "nemo_oracle_add_neuron_type": (i, [vp, C.c_char_p, C.POINTER(C.c_uint)]),
                "nemo_oracle_add_neurons": (i, [vp, C.c_uint, sz, u32p, C.c_uint, f32p]),
                "nemo_oracle_add_synapses": (i, [vp, sz, u32p, u32p, u32p, f32p, u8p, u64p]),
                "nemo_oracle_neuron_count": (i, [vp, C.POINTER(C.c_uint)]),
                "nemo_oracle_new_simulation": (vp, [vp, vp]),
                "nemo_oracle_delete_simulation": (None, [vp]),
                "nemo_oracle_step": (i, [vp, u32p, sz, u32p, f32p, sz, C.POINTER(C.POINTER(C.c_uint)), C.POINTER(sz)]),
                "nemo_oracle_run": (i, [vp, C.c_uint, C.c_uint, C.c_float, u32p, u32p, sz, C.POINTER(sz)]),
                "nemo_oracle_apply_stdp": (i, [vp, C.c_float]),
                "nemo_oracle_get_neuron_state": (i, [vp, C.c_uint, C.c_uint, C.POINTER(C.c_float)]),
                "nemo_oracle_get_neuron_parameter": (i, [vp, C.c_uint, C.c_uint, C.POINTER(C.c_float)]),
                "nemo_oracle_get_membrane_potential": (i, [vp, C.c_uint, C.POINTER(C.c_float)]),
                "nemo_oracle_set_neuron_state": (i, [vp, C.c_uint, C.c_uint, C.c_float]),
                "nemo_oracle_set_neuron_parameter": (i, [vp, C.c_uint, C.c_uint, C.c_float]),
                "nemo_oracle_set_neuron": (i, [vp, C.c_uint, C.c_uint, f32p]),
                "nemo_oracle_get_synapses_from": (i, [vp, C.c_uint, C.POINTER(C.POINTER(C.c_uint64)), C.POINTER(sz)]),
                "nemo_oracle_get_synapse_target": (i, [vp, C.c_uint64, C.POINTER(C.c_uint)]),
                "nemo_oracle_get_synapse_delay": (i, [vp, C.c_uint64, C.POINTER(C.c_uint)]),
                "nemo_oracle_get_synapse_weight": (i, [vp, C.c_uint64, C.POINTER(C.c_float)]),
                "nemo_oracle_get_synapse_plastic": (i, [vp, C.c_uint64, C.POINTER(C.c_ubyte)]),
                "nemo_oracle_get_all_weights_fx": (i, [vp, i32p, sz, C.POINTER(sz)]),
                "nemo_oracle_get_type_state": (i, [vp, C.c_uint, f32p, sz, C.POINTER(sz)]),
                "nemo_oracle_elapsed_simulation": (i, [vp, C.POINTER(C.c_ulong)]),
                "nemo_oracle_reset_timer": (i, [vp]),
                "nemo_oracle_urand": (C.c_uint, [u32p]),
                "nemo_oracle_nrand": (C.c_float, [u32p]),
                "nemo_oracle_seed_states": (None, [C.c_uint, C.c_uint, u32p]),
                "nemo_oracle_example_random": (i, [C.POINTER(vp), C.c_uint, C.c_uint, C.c_uint, C.c_int]),
                "nemo_oracle_example_random_ex": (i, [C.POINTER(vp), C.c_uint, C.c_uint, C.c_uint, C.c_int, C.c_uint,
                                                      C.c_float, C.c_float]),
                "nemo_oracle_network_synapse_count": (sz, [vp]),
                "nemo_oracle_network_synapses": (i, [vp, sz, u32p, u32p, u32p, f32p, u8p, C.POINTER(sz)]),
            }
            for name, (res, args) in sig.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def _check(code: int):
    if code != 0:
        raise NemoError(code, lib().nemo_oracle_strerror().decode())


def _u32(x):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.uint32)))


def _f32(x):
    return np.ascontiguousarray(np.atleast_1d(np.asarray(x, dtype=np.float32)))


class Configuration:
    """Mirror of nemo::Configuration (src/nemo/Configuration.hpp)."""

    def __init__(self):
        self._h = lib().nemo_oracle_new_configuration()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().nemo_oracle_delete_configuration(self._h)
            self._h = None

    def set_stdp_function(self, prefire, postfire, *limits):
        """(pre, post, minWeight, maxWeight) or (pre, post, minE, maxE, minI, maxI)
        -- the two overloads of Configuration::setStdpFunction
        (src/nemo/Configuration.cpp:80-100)."""
        if len(limits) == 2:
            min_w, max_w = limits
            limits = (0.0, max_w, 0.0, min_w)
        pre, post = _f32(prefire), _f32(postfire)
        _check(lib().nemo_oracle_set_stdp_function(self._h, pre, len(pre), post, len(post), *[float(v) for v in limits]))

    def set_write_only_synapses(self):
        _check(lib().nemo_oracle_set_write_only_synapses(self._h))

    def set_cuda_backend(self, device=-1):  # the oracle is CPU only
        pass

    def set_cpu_backend(self):
        pass


class Network:
    """Mirror of nemo::Network (src/nemo/Network.hpp)."""

    def __init__(self, _handle=None):
        self._h = _handle if _handle is not None else lib().nemo_oracle_new_network()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().nemo_oracle_delete_network(self._h)
            self._h = None

    def add_neuron_type(self, name: str) -> int:
        t = C.c_uint()
        _check(lib().nemo_oracle_add_neuron_type(self._h, name.encode(), C.byref(t)))
        return t.value

    def add_neuron(self, ntype: int, idx, *args):
        """add_neuron(type, idx, p0, p1, ..., s0, s1, ...); idx and the
        arguments may be scalars or equal-length vectors."""
        idx = _u32(idx)
        n = len(idx)
        cols = [np.broadcast_to(_f32(a), (n,)) for a in args]
        mat = np.ascontiguousarray(np.stack(cols, axis=1) if cols else np.zeros((n, 0), np.float32), dtype=np.float32)
        _check(lib().nemo_oracle_add_neurons(self._h, ntype, n, idx, len(args), mat.reshape(-1) if mat.size else np.zeros(1, np.float32)))

    def add_synapse(self, source, target, delay, weight, plastic):
        src, tgt, dly = _u32(source), _u32(target), _u32(delay)
        w = _f32(weight)
        pl = np.ascontiguousarray(np.atleast_1d(np.asarray(plastic, dtype=np.uint8)))
        n = max(len(src), len(tgt), len(dly), len(w), len(pl))
        src, tgt, dly, w, pl = (np.ascontiguousarray(np.broadcast_to(a, (n,))) for a in (src, tgt, dly, w, pl))
        ids = np.zeros(n, np.uint64)
        _check(lib().nemo_oracle_add_synapses(self._h, n, src, tgt, dly, w, pl, ids))
        return ids if n != 1 or np.ndim(source) else int(ids[0])

    def neuron_count(self) -> int:
        c = C.c_uint()
        _check(lib().nemo_oracle_neuron_count(self._h, C.byref(c)))
        return c.value

    def synapses(self):
        """All synapses in insertion order as numpy arrays."""
        L = lib()
        n = L.nemo_oracle_network_synapse_count(self._h)
        out = [np.zeros(n, np.uint32), np.zeros(n, np.uint32), np.zeros(n, np.uint32),
               np.zeros(n, np.float32), np.zeros(n, np.uint8)]
        ln = C.c_size_t()
        _check(L.nemo_oracle_network_synapses(self._h, n, *out, C.byref(ln)))
        return out


def example_random(ncount: int, scount: int, dmax: int, stdp: bool, seed: int | None = None,
                   sigma_exc: float = 5.0, sigma_inh: float = 2.0) -> Network:
    """The reference's random::construct (src/examples/random.cpp:63-88)."""
    h = C.c_void_p()
    _check(lib().nemo_oracle_example_random_ex(C.byref(h), ncount, scount, dmax, int(stdp),
                                               5489 if seed is None else seed, sigma_exc, sigma_inh))
    return Network(h.value)


class Simulation:
    """Mirror of nemo::Simulation on the reference CPU backend."""

    def __init__(self, net: Network, conf: Configuration):
        h = lib().nemo_oracle_new_simulation(net._h, conf._h)
        if not h:
            raise NemoError(6, lib().nemo_oracle_strerror().decode())
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().nemo_oracle_delete_simulation(self._h)
            self._h = None

    def step(self, fstim=None, istim=None):
        L = lib()
        f = _u32(fstim if fstim is not None else [])
        if istim:
            inid = _u32([p[0] for p in istim])
            icur = _f32([p[1] for p in istim])
        else:
            inid, icur = np.zeros(0, np.uint32), np.zeros(0, np.float32)
        fired = C.POINTER(C.c_uint)()
        n = C.c_size_t()
        _check(L.nemo_oracle_step(self._h, f if len(f) else np.zeros(1, np.uint32), len(f),
                                  inid if len(inid) else np.zeros(1, np.uint32),
                                  icur if len(icur) else np.zeros(1, np.float32), len(inid),
                                  C.byref(fired), C.byref(n)))
        return [fired[i] for i in range(n.value)]

    def run(self, steps: int, stdp_period: int = 0, reward: float = 1.0, max_ids: int | None = None):
        """Run `steps` unstimulated steps; returns (per-step counts, fired ids)."""
        counts = np.zeros(steps, np.uint32)
        cap = max_ids if max_ids is not None else steps * 4096
        ids = np.zeros(max(cap, 1), np.uint32)
        ln = C.c_size_t()
        _check(lib().nemo_oracle_run(self._h, steps, stdp_period, reward, counts, ids, cap, C.byref(ln)))
        return counts, ids[: ln.value].copy()

    def apply_stdp(self, reward: float):
        _check(lib().nemo_oracle_apply_stdp(self._h, float(reward)))

    def _getf(self, fn, *args):
        v = C.c_float()
        _check(fn(self._h, *args, C.byref(v)))
        return v.value

    def get_neuron_state(self, idx, var):
        return self._getf(lib().nemo_oracle_get_neuron_state, idx, var)

    def get_neuron_parameter(self, idx, p):
        return self._getf(lib().nemo_oracle_get_neuron_parameter, idx, p)

    def get_membrane_potential(self, idx):
        return self._getf(lib().nemo_oracle_get_membrane_potential, idx)

    def set_neuron_state(self, idx, var, val):
        _check(lib().nemo_oracle_set_neuron_state(self._h, idx, var, float(val)))

    def set_neuron_parameter(self, idx, p, val):
        _check(lib().nemo_oracle_set_neuron_parameter(self._h, idx, p, float(val)))

    def set_neuron(self, idx, *args):
        a = _f32(args)
        _check(lib().nemo_oracle_set_neuron(self._h, idx, len(a), a))

    def get_synapses_from(self, source):
        p = C.POINTER(C.c_uint64)()
        n = C.c_size_t()
        _check(lib().nemo_oracle_get_synapses_from(self._h, source, C.byref(p), C.byref(n)))
        return [p[i] for i in range(n.value)]

    def get_synapse_target(self, sid):
        v = C.c_uint()
        _check(lib().nemo_oracle_get_synapse_target(self._h, sid, C.byref(v)))
        return v.value

    def get_synapse_delay(self, sid):
        v = C.c_uint()
        _check(lib().nemo_oracle_get_synapse_delay(self._h, sid, C.byref(v)))
        return v.value

    def get_synapse_weight(self, sid):
        return self._getf(lib().nemo_oracle_get_synapse_weight, C.c_uint64(sid))

    def get_synapse_plastic(self, sid):
        v = C.c_ubyte()
        _check(lib().nemo_oracle_get_synapse_plastic(self._h, sid, C.byref(v)))
        return bool(v.value)

    def weights_fx(self, nsyn: int) -> np.ndarray:
        """All weights (raw Q11.20) in network iteration order."""
        out = np.zeros(max(nsyn, 1), np.int32)
        ln = C.c_size_t()
        _check(lib().nemo_oracle_get_all_weights_fx(self._h, out, len(out), C.byref(ln)))
        return out[: ln.value]

    def type_state(self, ntype: int, nstate: int, n: int) -> np.ndarray:
        out = np.zeros(max(nstate * n, 1), np.float32)
        ln = C.c_size_t()
        _check(lib().nemo_oracle_get_type_state(self._h, ntype, out, len(out), C.byref(ln)))
        return out[: ln.value].reshape(nstate, n) if ln.value else np.zeros((nstate, 0), np.float32)

    def elapsed_simulation(self):
        v = C.c_ulong()
        _check(lib().nemo_oracle_elapsed_simulation(self._h, C.byref(v)))
        return v.value

    def reset_timer(self):
        _check(lib().nemo_oracle_reset_timer(self._h))


def urand(state: np.ndarray) -> int:
    return lib().nemo_oracle_urand(state)


def nrand(state: np.ndarray) -> float:
    return lib().nemo_oracle_nrand(state)


def seed_states(first: int, count: int) -> np.ndarray:
    out = np.zeros(4 * max(count, 1), np.uint32)
    lib().nemo_oracle_seed_states(first, count, out)
    return out[: 4 * count].reshape(count, 4)
