"""ctypes binding of libb2b.so (include/b2b.h).

The library is loaded from the package directory.  There is no fallback: if libb2b.so is
missing or fails to load, importing the binding raises, so a machine with a GPU never runs
anything but the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libb2b.so")

B2B_OK = 0
STATUS_NAMES = {
    0: "B2B_OK", 1: "B2B_ERR_INVALID_ARG", 2: "B2B_ERR_OOM", 3: "B2B_ERR_QUEUE_OVERFLOW",
    4: "B2B_ERR_TIMEOUT", 5: "B2B_ERR_CUDA", 6: "B2B_ERR_STATE", 7: "B2B_ERR_UNSUPPORTED",
    8: "B2B_ERR_INDEX",
}
F32, F64 = 1, 2
NET_NO_GRAPH, NET_CHECKED, NET_RESET_BEFORE_SYNAPSES, NET_TWO_LAUNCH, NET_SMALL = 1, 2, 4, 8, 16
NET_PER_STEP = 32
NET_ONE_LAUNCH = 64
EFFECT_ADD, EFFECT_STDP = 1, 2
VARS = {"v": 0, "ge": 1, "gi": 2, "m": 3, "h": 4, "n": 5, "lastspike": 6,
        "not_refractory": 7}
SYN_VARS = {"i": 0, "j": 1, "delay": 2, "w": 3, "Apre": 4, "Apost": 5, "lastupdate": 6}
HINES_VARS = {"v": 0, "m": 1, "h": 2, "n": 3, "Ic": 4}


class B2BError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {message}" if message else name)


class Config(C.Structure):
    _fields_ = [("dt", C.c_double), ("device", C.c_int32), ("steps_per_graph", C.c_int32),
                ("seed", C.c_uint64), ("stream", C.c_void_p), ("flags", C.c_int32),
                ("reserved", C.c_int32)]


class LifParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("El", "taum", "taue", "taui", "ke", "ki", "Vt", "Vr", "refractory")] + \
               [(n, C.c_int32) for n in
                ("has_threshold", "has_reset", "unless_refractory", "reserved")]


class HhParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("Cm", "gl", "El", "EK", "ENa", "gNa", "gK", "VT", "Ee", "Ei", "taue", "taui",
                 "Vthr", "refractory")]


class StdpParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("taupre", "taupost", "dApre", "dApost", "wmin", "wmax")] + \
               [("pre_adds_weight", C.c_int32), ("reserved", C.c_int32)]


class HinesParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("Cm", "Ri", "El", "EK", "ENa", "gl", "gNa", "gK", "Vthr")] + \
               [("channel_dtype", C.c_int32), ("reserved", C.c_int32)]


class TuneResult(C.Structure):
    _fields_ = [("site_kind", C.c_int32), ("site_index", C.c_int32), ("choice_a", C.c_int32),
                ("choice_b", C.c_int32), ("best_ms", C.c_double), ("default_ms", C.c_double)]


P = C.c_void_p
I32, I64, U64, DBL = C.c_int32, C.c_int64, C.c_uint64, C.c_double
PI32, PI64 = C.POINTER(C.c_int32), C.POINTER(C.c_int64)

# name: (restype, argtypes) — one entry per declaration of include/b2b.h
PROTOTYPES = {
    "b2b_create": (I32, [C.POINTER(Config), C.POINTER(P)]),
    "b2b_destroy": (I32, [P]),
    "b2b_last_error": (I32, [P, C.c_char_p, C.c_size_t]),
    "b2b_status_string": (C.c_char_p, [I32]),
    "b2b_abi_version": (I32, []),
    "b2b_group_lif": (I32, [P, I64, I32, C.POINTER(LifParams), PI32]),
    "b2b_group_hh": (I32, [P, I64, I32, C.POINTER(HhParams), PI32]),
    "b2b_group_poisson": (I32, [P, I64, I32, DBL, PI32]),
    "b2b_group_spikegen": (I32, [P, I64, I64, P, P, PI32]),
    "b2b_spikemon_get_range": (I32, [P, I32, I64, I64, PI64, P, P, I64]),
    "b2b_spikegen_period": (I32, [P, I32, I64]),
    "b2b_timedarray": (I32, [P, I32, P, I64, I64, DBL]),
    "b2b_poisson_input": (I32, [P, I32, I32, I64, DBL, DBL, PI32]),
    "b2b_state_set": (I32, [P, I32, I32, P, I64]),
    "b2b_state_get": (I32, [P, I32, I32, P, I64]),
    "b2b_state_ptr": (I32, [P, I32, I32, C.POINTER(P), PI64]),
    "b2b_synapses": (I32, [P, I32, I32, I32, I32, I64, P, P, P, DBL, P, I32,
                           C.POINTER(StdpParams), PI32]),
    "b2b_synapses_random": (I32, [P, I32, I32, I32, I32, I32, DBL, I32, I32, DBL, U64, PI32]),
    "b2b_connect_random_static": (I32, [I32, P, I32, I32, I32, DBL, I32, I32, U64, P, P, P, I64,
                                        PI64]),
    "b2b_syn_count": (I32, [P, I32, PI64]),
    "b2b_syn_get": (I32, [P, I32, I32, P, I64]),
    "b2b_finalize": (I32, [P]),
    "b2b_run": (I32, [P, I64]),
    "b2b_sync": (I32, [P, PI32]),
    "b2b_store": (I32, [P, I32]),
    "b2b_restore": (I32, [P, I32]),
    "b2b_time": (I32, [P, PI64, C.POINTER(DBL)]),
    "b2b_kernel_launches": (I32, [P, PI64]),
    "b2b_run_mode": (I32, [P, PI32]),
    "b2b_profile": (I32, [P, I64, C.POINTER(DBL), PI32, I32, PI32]),
    "b2b_syn_set_delays": (I32, [P, I32, P, I64]),
    "b2b_wait_selftest": (I32, [I32, P, C.c_uint32, I32, PI32]),
    "b2b_recip_selftest": (I32, [I32, P, P, I64]),
    "b2b_group_model": (I32, [P, I64, I32, C.c_char_p, DBL, PI32]),
    "b2b_rng_normals_get": (I32, [P, I32, P, I64, I64]),
    "b2b_atomic_rate": (I32, [I32, P, I64, I64, I32, C.POINTER(DBL), C.POINTER(DBL),
                              C.POINTER(DBL)]),
    "b2b_profile_graph": (I32, [P, I64, C.POINTER(DBL), PI32, I32, PI32, C.POINTER(DBL)]),
    "b2b_spikemon": (I32, [P, I32, I64]),
    "b2b_spikemon_get": (I32, [P, I32, PI64, P, P, I64]),
    "b2b_spikemon_fetch": (I32, [P, I32, I64, PI64, PI64, P, P, I64]),
    "b2b_spikes_last": (I32, [P, I32, PI64, P, I64]),
    "b2b_queue_get": (I32, [P, I32, PI64, P, P, P, I64]),
    "b2b_rng_uniforms_get": (I32, [P, I32, P, I64, I64]),
    "b2b_hines_create": (I32, [P, I32, P, P, P, P, P, P, P, C.POINTER(HinesParams),
                               C.POINTER(P)]),
    "b2b_hines_set_current": (I32, [P, P]),
    "b2b_hines_state_set": (I32, [P, I32, P, I64]),
    "b2b_hines_state_get": (I32, [P, I32, P, I64]),
    "b2b_hines_run": (I32, [P, I64]),
    "b2b_hines_spike_counts": (I32, [P, P, I32]),
    "b2b_hines_destroy": (I32, [P]),
    "b2b_autotune": (I32, [P, I32, C.POINTER(TuneResult), I32, PI32]),
    "b2b_out_degree": (I32, [P, I32, P, I64]),
    "b2b_tune_apply": (I32, [P, C.POINTER(TuneResult), I32]),
    "b2b_spikemon_fetch_population": (I32, [P, I32, I64, PI64, PI64, P, P, I64]),
    "b2b_group_offset": (I32, [P, I32, PI64]),
    "b2b_statemon": (I32, [P, I32, I32, PI64, I64, I32, I64, PI32]),
    "b2b_statemon_get": (I32, [P, I32, PI64, PI64, P, I64]),
    "b2b_ratemon": (I32, [P, I32, I64, PI32]),
    "b2b_ratemon_get": (I32, [P, I32, PI64, PI64, PI32, I64]),
    "b2b_mlp_create": (I32, [I32, P, U64, C.POINTER(P)]),
    "b2b_mlp_destroy": (I32, [P]),
    "b2b_mlp_params_get": (I32, [P, P, I64]),
    "b2b_mlp_params_set": (I32, [P, P, I64]),
    "b2b_mlp_scaling_get": (I32, [P, P]),
    "b2b_mlp_scaling_set": (I32, [P, P]),
    "b2b_mlp_fit_scaling": (I32, [P, P, P, I64]),
    "b2b_mlp_forward": (I32, [P, P, P, I64, I32]),
    "b2b_mlp_grad": (I32, [P, P, P, I64, P, I64, C.POINTER(DBL)]),
    "b2b_mlp_train": (I32, [P, P, P, I64, I32, I32, DBL, P]),
    "b2b_hh_gating_exact": (I32, [C.POINTER(HhParams), DBL, P, P, I64, I32, P]),
    "b2b_hh_gating_sample": (I32, [P, I32, P, I64]),
    "b2b_group_hh_surrogate": (I32, [P, I32, P, DBL, I32]),
    "b2b_surrogate_stats": (I32, [P, I32, PI64, PI64]),
}
MLP_NPARAMS = 4675

_lib = None


def lib() -> C.CDLL:
    """Loads libb2b.so once; raises if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(
                f"{_LIB_PATH} is missing; build it with `python -m brian2cuda_b200.build`")
        handle = C.CDLL(_LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def lib_path() -> str:
    return _LIB_PATH
