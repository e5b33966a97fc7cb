"""ctypes binding of ``libstarmap_gpu.so`` (the C ABI of include/starmap_gpu.h).

The shared object is loaded from the package directory.  There is no CPU
fallback: if the library is missing or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstarmap_gpu.so")

SMG_OK = 0
SMG_EINVAL = -1
SMG_ECUDA = -2
SMG_ETIMEOUT = -3
SMG_ENONFINITE = -4
SMG_ENOMEM = -5
SMG_ESTATE = -6

# smg_tune keys
SMG_TUNE_PAIR_GROUP = 1
SMG_TUNE_PAIR_BLOCK = 2
SMG_TUNE_PAIR_UNROLL = 3
SMG_TUNE_PAIR_MINB = 4
SMG_TUNE_ADJ_FUSED = 5
SMG_TUNE_JIT_BLOCK = 6
SMG_TUNE_JIT_GROUP = 7
SMG_TUNE_JIT_REGS = 8
SMG_TUNE_JIT_SPLIT = 9
SMG_TUNE_JIT_CALLS = 10
SMG_TUNE_JIT_XPAIR = 11
SMG_TUNE_JIT_PREFETCH = 12
SMG_TUNE_JIT_BAND = 13
SMG_TUNE_JIT_CONST = 14
SMG_TUNE_GRAPH_STEPS = 15
SMG_TUNE_JIT_STAGED = 16
SMG_TUNE_JIT_SLICES = 17
SMG_TUNE_JIT_STAGES = 18
SMG_TUNE_JIT_ROWS = 19
SMG_TUNE_ADJ_PRIORITY = 20
SMG_TUNE_DIRECT_XFER = 21
SMG_TUNE_JIT_LANES = 22

# smg_check_expr kinds
SMG_EXPR_SOURCE, SMG_EXPR_MATERIAL, SMG_EXPR_FILTER = 0, 1, 2

SMG_VARIANT_AUTO = 0
SMG_VARIANT_GENERIC = 1
SMG_VARIANT_STRIP = 2
SMG_VARIANT_STAGED = 3
SMG_VARIANT_PAIR = 4
SMG_VARIANT_JIT = 5
_NAMES = {SMG_EINVAL: "SMG_EINVAL", SMG_ECUDA: "SMG_ECUDA", SMG_ETIMEOUT: "SMG_ETIMEOUT",
          SMG_ENONFINITE: "SMG_ENONFINITE", SMG_ENOMEM: "SMG_ENOMEM", SMG_ESTATE: "SMG_ESTATE"}

FILTER_NONE, FILTER_SUBSTEP, FILTER_FULL = 0, 1, 2


class SmgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


class smg_field(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_double)), ("scalar", C.c_double), ("grid", C.c_int32 * 3)]


class smg_problem(C.Structure):
    _fields_ = [
        ("n_sys", C.c_int32), ("n", C.c_int32 * 3), ("bc", C.c_int32 * 3), ("h", C.c_double * 3),
        ("gt", C.POINTER(C.c_int32)),
        ("Mx", C.POINTER(C.c_double)), ("My", C.POINTER(C.c_double)), ("Mz", C.POINTER(C.c_double)),
        ("n_fields", C.c_int32), ("fields", C.POINTER(smg_field)),
        ("sigma_t", C.POINTER(C.c_int32)), ("decay_t", C.POINTER(C.c_int32)),
        ("sigma_a", C.c_int32), ("decay_a", C.c_int32),
        ("source", C.POINTER(C.c_int32)),
        ("filter_mode", C.c_int32),
        ("filter1", C.POINTER(C.c_int32)), ("filter2", C.POINTER(C.c_int32)),
    ]


_lib = None

# name -> (restype, argtypes); every symbol declared in include/starmap_gpu.h
SIGNATURES = {
    "smg_version": (C.c_char_p, []),
    "smg_last_error": (C.c_char_p, [C.c_void_p]),
    "smg_device_count": (C.c_int, []),
    "smg_set_device": (C.c_int, [C.c_int32]),
    "smg_create": (C.c_int, [C.POINTER(smg_problem), C.POINTER(C.c_void_p)]),
    "smg_destroy": (None, [C.c_void_p]),
    "smg_set_state": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_double))]),
    "smg_get_state": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_double))]),
    "smg_set_field": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_double]),
    "smg_set_dt": (C.c_int, [C.c_void_p, C.c_double]),
    "smg_set_time": (C.c_int, [C.c_void_p, C.c_double]),
    "smg_snapshot": (C.c_int, [C.c_void_p]),
    "smg_get_interp": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.POINTER(C.c_double))]),
    "smg_set_filter_expr": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.POINTER(C.c_int32),
                                      C.POINTER(C.POINTER(C.c_double))]),
    "smg_set_material_expr": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int32,
                                        C.POINTER(C.c_int32), C.c_int32, C.c_int32,
                                        C.POINTER(C.POINTER(C.c_double))]),
    "smg_check_expr": (C.c_int, [C.c_int32, C.c_char_p]),
    "smg_set_source_expr": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "smg_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "smg_sync": (C.c_int, [C.c_void_p]),
    "smg_set_variant": (C.c_int, [C.c_void_p, C.c_int32]),
    "smg_tune": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "smg_last_run_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "smg_layout": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "smg_check_finite": (C.c_int, [C.c_void_p]),
    "smg_state_sumsq": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "smg_sumsq_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]),
    "smg_classify": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "smg_forward": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64]),
    "smg_misfit": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "smg_adjoint_seed": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_double))]),
    "smg_backward": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_double))]),
    "smg_adjoint_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "smg_adjoint_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "smg_active_variant": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_char_p, C.c_int64]),
    "smg_jit_stats": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "smg_growth_radius": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "smg_jit_source": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32, C.c_int32,
                                 C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]),
    "smg_batch_create": (C.c_int, [C.c_int32, C.POINTER(C.POINTER(smg_problem)), C.POINTER(C.c_void_p)]),
    "smg_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "smg_batch_destroy": (None, [C.c_void_p]),
    "smg_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "smg_batch_instance": (C.c_void_p, [C.c_void_p, C.c_int32]),
    "smg_batch_set_dt": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "smg_batch_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "smg_batch_last_run_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "smg_batch_tune": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64]),
    "smg_batch_config": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "smg_batch_autotune": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_double)]),
}


def lib():
    """Load the library (once).  Raises if it is absent: the product has no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m starmap_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, handle=None):
    if code < 0:
        msg = lib().smg_last_error(handle)
        raise SmgError(code, msg.decode() if msg else "")
    return code


def check_batch(code: int, batch=None):
    if code < 0:
        msg = lib().smg_batch_last_error(batch)
        raise SmgError(code, msg.decode() if msg else "")
    return code


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def classify(Mx, My, Mz) -> np.ndarray:
    """Grid types (n_sys, 3) in {1, 2} via the library's smg_classify."""
    n = Mz.shape[0]
    mats = [np.asfortranarray(np.asarray(M, dtype=np.float64)) for M in (Mx, My, Mz)]
    out = np.zeros(3 * n, dtype=np.int32)
    check(lib().smg_classify(n, dptr(mats[0]), dptr(mats[1]), dptr(mats[2]), iptr(out)))
    return out.reshape(n, 3)
