"""ctypes binding of the C ABI in include/pt_gravity.h (libpt_gravity.so).

There is no fallback: if the CUDA library is missing or cannot be loaded, the
import of the binding raises.  Build it with ``python -m paratreet_b200.build``
(or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpt_gravity.so")

PT_OK = 0
PT_FP64, PT_MIXED, PT_FP64_LISTS = 0, 1, 2
PT_KKD, PT_KDK = 0, 1
PT_TRANSPOSED_DOWN, PT_BASIC_DOWN = 0, 1

ERRORS = {
    -1: "PT_E_ARG", -2: "PT_E_CUDA", -3: "PT_E_NOMEM", -4: "PT_E_STATE",
    -5: "PT_E_DEVICE", -6: "PT_E_NONFINITE", -7: "PT_E_UNSUPPORTED",
}


class PtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class PtConfig(C.Structure):
    _fields_ = [
        ("theta", C.c_double),
        ("bucket", C.c_int),
        ("precision", C.c_int),
        ("integrator", C.c_int),
        ("dt_max", C.c_double),
        ("device", C.c_int),
        ("record_lists", C.c_int),
        ("periodic", C.c_int),
        ("n_replicas", C.c_int),
        ("period", C.c_double),
        ("ewald_rcut", C.c_double),
        ("ewald_hcut", C.c_double),
        ("traversal", C.c_int),
        ("reserved", C.c_int * 7),
    ]


class PtCounters(C.Structure):
    _fields_ = [
        ("n_pp", C.c_uint64),
        ("n_pc", C.c_uint64),
        ("n_open", C.c_uint64),
        ("n_nodes", C.c_int64),
        ("n_buckets", C.c_int64),
        ("depth", C.c_int32),
        ("launches", C.c_int32),
        ("ms_keys", C.c_float),
        ("ms_sort", C.c_float),
        ("ms_build", C.c_float),
        ("ms_upward", C.c_float),
        ("ms_traverse", C.c_float),
        ("ms_total", C.c_float),
    ]


# Every exported entry point: name -> (restype, argtypes).
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_i64 = C.c_int64
SIGNATURES = {
    "pt_abi_version": (C.c_int, []),
    "pt_config_default": (C.c_int, [C.POINTER(PtConfig)]),
    "pt_create": (C.c_int, [C.POINTER(PtConfig), C.POINTER(_vp)]),
    "pt_destroy": (C.c_int, [_vp]),
    "pt_last_error": (C.c_char_p, [_vp]),
    "pt_set_stream": (C.c_int, [_vp, _vp]),
    "pt_set_theta": (C.c_int, [_vp, C.c_double]),
    "pt_set_precision": (C.c_int, [_vp, C.c_int]),
    "pt_set_sort_spin_limit": (C.c_int, [_vp, _i64]),
    "pt_set_list_region": (C.c_int, [_vp, _i64]),
    "pt_set_particles": (C.c_int, [_vp, _i64] + [_vp] * 8),
    "pt_set_particles_device": (C.c_int, [_vp, _i64] + [_vp] * 8),
    "pt_num_particles": (_i64, [_vp]),
    "pt_compute_forces": (C.c_int, [_vp]),
    "pt_compute_forces_range": (C.c_int, [_vp, _i64, _i64]),
    "pt_get_accel": (C.c_int, [_vp] + [_vp] * 5),
    "pt_device_accel": (C.c_int, [_vp] + [C.POINTER(_vp)] * 6),
    "pt_step": (C.c_int, [_vp, C.c_int]),
    "pt_get_state": (C.c_int, [_vp] + [_vp] * 6),
    "pt_last_dt": (C.c_int, [_vp, _dp]),
    "pt_get_keys": (C.c_int, [_vp, _vp]),
    "pt_get_universe": (C.c_int, [_vp, _vp, _vp]),
    "pt_get_tree_size": (C.c_int, [_vp, C.POINTER(_i64), C.POINTER(_i64)]),
    "pt_get_tree": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pt_get_bucket_keys": (C.c_int, [_vp, _vp]),
    "pt_get_lists_size": (C.c_int, [_vp, C.POINTER(_i64)]),
    "pt_get_lists": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pt_get_list_digests": (C.c_int, [_vp, C.c_int, _vp, _vp]),
    "pt_get_counters": (C.c_int, [_vp, C.POINTER(PtCounters)]),
    "pt_direct_sum": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "pt_ewald_direct_sum": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "pt_advance": (C.c_int, [_vp, _vp]),
    "pt_sph_density": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "pt_sph_pressure": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pt_sph_step": (C.c_int, [_vp, C.c_int] + [_vp] * 5),
    "pt_get_bucket_work": (C.c_int, [_vp, _vp]),
    "pt_forces_frozen": (C.c_int, [_vp] + [_vp] * 4),
    "pt_adjoint": (C.c_int, [_vp] + [_vp] * 7),
    "pt_chain_grad": (C.c_int, [_vp, C.c_int, C.c_double, C.c_int] + [_vp] * 3 + [_vp] * 8),
    "pt_direct_sum_noalloc": (C.c_int, [_i64] + [_vp] * 5 + [_i64] + [_vp] * 6 + [C.c_char_p, C.c_size_t]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load libpt_gravity.so and bind every entry point (raises if missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build the CUDA library (python -m paratreet_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)
