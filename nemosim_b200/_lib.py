"""Loader of the native library (``lib/libnemo_b200.so``) and its C ABI
signatures (``include/nemo_b200.h``).

There is no fallback: if the library is missing and cannot be built, or a
symbol is missing, importing the bindings raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

_lock = threading.Lock()
_lib = None

u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
vp, st, sz = C.c_void_p, C.c_int, C.c_size_t
PU = C.POINTER(C.c_uint)
PF = C.POINTER(C.c_float)

# name -> (restype, argtypes); every entry point of include/nemo_b200.h
SIGNATURES = {
    "nemo_version": (C.c_char_p, []),
    "nemo_add_plugin_path": (st, [C.c_char_p]),
    "nemo_cuda_device_count": (st, [PU]),
    "nemo_cuda_device_description": (st, [C.c_uint, C.POINTER(C.c_char_p)]),
    "nemo_new_configuration": (vp, []),
    "nemo_delete_configuration": (None, [vp]),
    "nemo_log_stdout": (st, [vp]),
    "nemo_set_stdp_function": (st, [vp, f32p, sz, f32p, sz, C.c_float, C.c_float, C.c_float, C.c_float]),
    "nemo_set_cpu_backend": (st, [vp]),
    "nemo_set_cuda_backend": (st, [vp, C.c_int]),
    "nemo_cuda_device": (st, [vp, C.POINTER(C.c_int)]),
    "nemo_backend": (st, [vp, PU]),
    "nemo_backend_description": (st, [vp, C.POINTER(C.c_char_p)]),
    "nemo_set_write_only_synapses": (st, [vp]),
    "nemo_new_network": (vp, []),
    "nemo_delete_network": (None, [vp]),
    "nemo_add_neuron_type": (st, [vp, C.c_char_p, PU]),
    "nemo_add_neuron_iz": (st, [vp, C.c_uint] + [C.c_float] * 7),
    "nemo_add_neuron": (st, [vp, C.c_uint, C.c_uint, C.c_uint, f32p]),
    "nemo_add_synapse": (st, [vp, C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_ubyte, C.POINTER(C.c_uint64)]),
    "nemo_neuron_count": (st, [vp, PU]),
    "nemo_new_simulation": (vp, [vp, vp]),
    "nemo_delete_simulation": (None, [vp]),
    "nemo_step": (st, [vp, u32p, sz, u32p, f32p, sz, C.POINTER(PU), C.POINTER(sz)]),
    "nemo_b200_step_no_alloc": (st, [vp, u32p, sz, u32p, f32p, sz, u32p, sz, C.POINTER(sz)]),
    "nemo_apply_stdp": (st, [vp, C.c_float]),
    "nemo_get_membrane_potential": (st, [vp, C.c_uint, PF]),
    "nemo_get_neuron_state_n": (st, [vp, C.c_uint, C.c_uint, PF]),
    "nemo_get_neuron_parameter_n": (st, [vp, C.c_uint, C.c_uint, PF]),
    "nemo_get_neuron_state_s": (st, [vp, C.c_uint, C.c_uint, PF]),
    "nemo_get_neuron_parameter_s": (st, [vp, C.c_uint, C.c_uint, PF]),
    "nemo_get_synapse_source_n": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_source_s": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_target_n": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_target_s": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_delay_n": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_delay_s": (st, [vp, C.c_uint64, PU]),
    "nemo_get_synapse_weight_n": (st, [vp, C.c_uint64, PF]),
    "nemo_get_synapse_weight_s": (st, [vp, C.c_uint64, PF]),
    "nemo_get_synapse_plastic_n": (st, [vp, C.c_uint64, C.POINTER(C.c_ubyte)]),
    "nemo_get_synapse_plastic_s": (st, [vp, C.c_uint64, C.POINTER(C.c_ubyte)]),
    "nemo_get_synapses_from_n": (st, [vp, C.c_uint, C.POINTER(C.POINTER(C.c_uint64)), C.POINTER(sz)]),
    "nemo_get_synapses_from_s": (st, [vp, C.c_uint, C.POINTER(C.POINTER(C.c_uint64)), C.POINTER(sz)]),
    "nemo_set_neuron_n": (st, [vp, C.c_uint, C.c_uint, f32p]),
    "nemo_set_neuron_s": (st, [vp, C.c_uint, C.c_uint, f32p]),
    "nemo_set_neuron_iz_n": (st, [vp, C.c_uint] + [C.c_float] * 7),
    "nemo_set_neuron_iz_s": (st, [vp, C.c_uint] + [C.c_float] * 7),
    "nemo_set_neuron_state_n": (st, [vp, C.c_uint, C.c_uint, C.c_float]),
    "nemo_set_neuron_parameter_n": (st, [vp, C.c_uint, C.c_uint, C.c_float]),
    "nemo_set_neuron_state_s": (st, [vp, C.c_uint, C.c_uint, C.c_float]),
    "nemo_set_neuron_parameter_s": (st, [vp, C.c_uint, C.c_uint, C.c_float]),
    "nemo_elapsed_wallclock": (st, [vp, C.POINTER(C.c_ulong)]),
    "nemo_elapsed_simulation": (st, [vp, C.POINTER(C.c_ulong)]),
    "nemo_reset_timer": (st, [vp]),
    "nemo_strerror": (C.c_char_p, []),
    "cuda_device_count": (C.c_uint, []),
    "cuda_device_description": (C.c_char_p, [C.c_uint]),
    "nemo_b200_add_neurons": (st, [vp, C.c_uint, sz, u32p, C.c_uint, f32p]),
    "nemo_b200_add_synapses": (st, [vp, sz, u32p, u32p, u32p, f32p, u8p, u64p]),
    "nemo_b200_example_random": (st, [C.POINTER(vp), C.c_uint, C.c_uint, C.c_uint, C.c_int]),
    "nemo_b200_example_random_ex": (st, [C.POINTER(vp), C.c_uint, C.c_uint, C.c_uint, C.c_int, C.c_uint,
                                         C.c_float, C.c_float]),
    "nemo_b200_run": (st, [vp, C.c_uint, C.c_uint, C.c_float, vp, vp, vp, sz, C.POINTER(sz)]),
    "nemo_b200_new_batch": (vp, [C.POINTER(vp), C.c_uint, vp]),
    "nemo_b200_network_count": (st, [vp, PU]),
    "nemo_b200_batch_get_type_state": (st, [vp, C.c_uint, C.c_uint, f32p, sz, C.POINTER(sz)]),
    "nemo_b200_get_weights_fx": (st, [vp, i32p, sz, C.POINTER(sz)]),
    "nemo_b200_get_type_state": (st, [vp, C.c_uint, f32p, sz, C.POINTER(sz)]),
    "nemo_b200_synapse_count": (st, [vp, C.POINTER(C.c_uint64)]),
    "nemo_b200_set_profiling": (st, [vp, C.c_int]),
    "nemo_b200_set_graphs": (st, [vp, C.c_int]),
    "nemo_b200_set_persistent": (st, [vp, C.c_int]),
    "nemo_b200_set_resident_step": (st, [vp, C.c_uint]),
    "nemo_b200_set_wait_limit": (st, [vp, C.c_uint]),
    "nemo_b200_set_device_construction": (st, [vp, C.c_int]),
    "nemo_b200_bench_step_loop": (st, [vp, u32p, sz, C.c_uint, C.c_uint, C.c_float, C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_double)]),
    "nemo_b200_scatter_probe": (st, [C.c_uint, C.c_uint, C.c_int, C.c_uint, C.c_int, C.c_uint,
                                     C.POINTER(C.c_float)]),
    "nemo_b200_connectivity_digest": (st, [vp, u64p]),
    "nemo_b200_trace_phases": (st, [vp, C.c_uint, u64p, sz, PU]),

    "nemo_b200_run_stats": (st, [vp, PF, PF, PU] + [C.POINTER(C.c_uint64)] * 4),
    "nemo_b200_set_launch": (st, [vp, C.c_uint, C.c_uint]),
    "nemo_b200_get_launch": (st, [vp, PU, PU]),
    "nemo_b200_autotune": (st, [vp, C.c_uint, PF]),
    "nemo_b200_step_events": (st, [vp, C.POINTER(C.c_uint64)]),
    "nemo_b200_neuron_type_count": (C.c_uint, []),
    "nemo_b200_neuron_type_name": (C.c_char_p, [C.c_uint]),
    "nemo_b200_libm_calibration": (st, [C.POINTER(C.c_uint64)] * 3),
    "nemo_b200_libm_verify": (st, [C.POINTER(C.c_uint64)]),
    "nemo_b200_last_status": (st, []),
    "nemo_b200_bptt_new": (vp, [C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint, sz, u32p, u32p, u32p,
                                C.c_int, C.c_int]),
    "nemo_b200_bptt_delete": (None, [vp]),
    "nemo_b200_bptt_forward": (st, [vp] + [vp] * 8 + [vp]),
    "nemo_b200_bptt_backward": (st, [vp] + [vp] * 10 + [vp]),
    "nemo_b200_bptt_readout": (st, [vp, vp, vp]),
    "nemo_b200_host_nrand": (C.c_float, [u32p]),
}


def library_path() -> str:
    return _build.LIB


def lib():
    """The loaded native library (built first if it is missing or stale and
    nvcc is available)."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.LIB
            try:
                _build.build()
            except RuntimeError:
                if not os.path.exists(path):
                    raise
            if not os.path.exists(path):
                raise RuntimeError(f"native library {path} is missing; run nemosim_b200/build.py")
            L = C.CDLL(path)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)  # AttributeError if the ABI lacks a symbol
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib
