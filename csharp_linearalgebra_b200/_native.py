"""ctypes binding of libtensile_b200.so, the sm_100a CUDA library.

This is the binding a Python caller of the C ABI (include/tensile_b200.h)
writes; a C# caller binds the same symbols through NativeLibrary and unmanaged
function pointers. There is no fallback: if the library is missing or cannot
load, importing the package's compute API raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtensile_b200.so")

TNS_OK = 0
TNS_E_ARGUMENT = 1
TNS_E_SINGULAR = 2
TNS_E_ALLOCATION_LIMIT = 3
TNS_E_OUT_OF_MEMORY = 4
TNS_E_DEVICE = 5
TNS_E_TIMEOUT = 6
TNS_E_DISPOSED = 7
TNS_E_OUT_OF_RANGE = 8
TNS_E_NULL = 9
TNS_E_OPERATOR = 10


class LuInfo(C.Structure):
    _fields_ = [("singular_column", C.c_int), ("smallest_pivot", C.c_double),
                ("largest_pivot", C.c_double), ("one_norm", C.c_double)]


class NormestResult(C.Structure):
    _fields_ = [("value", C.c_double), ("iterations", C.c_int), ("products", C.c_int)]


class ExpmInfo(C.Structure):
    _fields_ = [("degree", C.c_int), ("squarings", C.c_int)]


class ExpmvInfo(C.Structure):
    _fields_ = [("degree", C.c_int), ("scaling", C.c_int), ("applications", C.c_int),
                ("early_exits", C.c_int)]


class MixedInfo(C.Structure):
    _fields_ = [("moduli", C.c_int), ("factorizations", C.c_int), ("iterations", C.c_int),
                ("backward_error", C.c_double), ("rcond", C.c_double), ("pivoting", C.c_int)]


class Stats(C.Structure):
    _fields_ = [("kernel_launches", C.c_longlong), ("gemm_launches", C.c_longlong),
                ("gemm_flops", C.c_double), ("gemm_ms", C.c_double), ("gemm_bytes", C.c_double),
                ("split_launches", C.c_longlong), ("split_flops", C.c_double), ("split_int8_ops", C.c_double),
                ("split_ms", C.c_double), ("split_bytes", C.c_double), ("autotune_trials", C.c_longlong),
                ("exact_fallbacks", C.c_longlong)]


class LuTimings(C.Structure):
    _fields_ = [("panel_ms", C.c_double), ("swaps_ms", C.c_double), ("triangular_ms", C.c_double),
                ("gemm_ms", C.c_double), ("total_ms", C.c_double), ("unattributed_ms", C.c_double),
                ("block_steps", C.c_longlong), ("factorizations", C.c_longlong)]


# y := A x on device panels: (user, ncols, x, y, ld, stream) -> status
APPLY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)

# name -> (restype, argtypes)
_P, _I, _D, _LL, _CH = C.c_void_p, C.c_int, C.c_double, C.c_longlong, C.c_char
SIGNATURES = {
    "tns_create": (_I, [_I, _LL, C.POINTER(_P)]),
    "tns_destroy": (_I, [_P]),
    "tns_last_error": (C.c_char_p, [_P]),
    "tns_set_max_elements": (_I, [_P, _LL]),
    "tns_dgemm": (_I, [_P, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "tns_dgemm_device": (_I, [_P, _I, _I, _I, _D, _P, _I, _P, _I, _D, _P, _I]),
    "tns_zgemm": (_I, [_P, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I]),
    "tns_zgemm_device": (_I, [_P, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I]),
    "tns_dgemm_split": (_I, [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I, _I]),
    "tns_zgemm_split": (_I, [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I, _I]),
    "tns_set_split_moduli": (_I, [_P, _I]),
    "tns_dnorm": (_I, [_P, _CH, _I, _I, _P, _I, C.POINTER(_D)]),
    "tns_znorm": (_I, [_P, _CH, _I, _I, _P, _I, C.POINTER(_D)]),
    "tns_dgetrf": (_I, [_P, _I, _I, _P, _I, _I, _P, C.POINTER(LuInfo)]),
    "tns_zgetrf": (_I, [_P, _I, _I, _P, _I, _I, _P, C.POINTER(LuInfo)]),
    "tns_dgetrs": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I, _I]),
    "tns_zgetrs": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I, _I]),
    **{name: (_I, [_P, _I, _I, _P, _I, _P, _I]) for name in (
        "tns_dsolve_upper", "tns_dsolve_upper_transposed", "tns_dsolve_lower", "tns_dsolve_lower_transposed",
        "tns_dsolve_lower_unit", "tns_dsolve_lower_unit_transposed", "tns_zsolve_upper", "tns_zsolve_upper_adjoint",
        "tns_zsolve_lower_unit", "tns_zsolve_lower_unit_adjoint")},
    **{name: (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I]) for name in (
        "tns_dmultiply_panel", "tns_dmultiply_panel_transposed", "tns_zmultiply_panel", "tns_zmultiply_panel_adjoint")},
    "tns_dgecon": (_I, [_P, _I, _P, _I, _P, _I, _D, C.POINTER(_D)]),
    "tns_zgecon": (_I, [_P, _I, _P, _I, _P, _I, _D, C.POINTER(_D)]),
    "tns_dnormest1_power": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, C.POINTER(NormestResult)]),
    "tns_znormest1_power": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, C.POINTER(NormestResult)]),
    "tns_dexpm": (_I, [_P, _I, _P, _I, _P, _I, C.POINTER(ExpmInfo)]),
    "tns_zexpm": (_I, [_P, _I, _P, _I, _P, _I, C.POINTER(ExpmInfo)]),
    "tns_zexpm_batched": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "tns_zexpm_batched_device": (_I, [_P, _I, _P, _P, _P, _P, _P, _P]),
    "tns_dexpmv": (_I, [_P, _I, _P, _I, _I, _P, _I, _D, _P, _I, C.POINTER(ExpmvInfo)]),
    "tns_zexpmv": (_I, [_P, _I, _P, _I, _I, _P, _I, _D, _P, _I, C.POINTER(ExpmvInfo)]),
    "tns_dexpmv_batched": (_I, [_P, _I, _P, _P, _P, _I, _P, _P, _D, _P, _P, _P]),
    "tns_zexpmv_batched": (_I, [_P, _I, _P, _P, _P, _I, _P, _P, _D, _P, _P, _P]),
    "tns_zexpmv_batched_device": (_I, [_P, _I, _P, _P, _P, _I, _P, _P, _D, _P, _P, _P]),
    "tns_zexpmv_select_batched": (_I, [_P, _I, _P, _P, _P, _I, _D, _P]),
    "tns_zexpmv_select_batched_device": (_I, [_P, _I, _P, _P, _P, _I, _D, _P]),
    "tns_dexpm_frechet": (_I, [_P, _I, _P, _I, _P, _I, _P, _I, _P, _I, C.POINTER(ExpmInfo)]),
    "tns_zexpm_frechet": (_I, [_P, _I, _P, _I, _P, _I, _P, _I, _P, _I, C.POINTER(ExpmInfo)]),
    "tns_dexpmv_gradient": (_I, [_P, _I, _I, _D, _P, _I, _P, _I, _P, _I, C.POINTER(_D), _P, _I, _P, _I,
                                 C.POINTER(_D), _P, _I, C.POINTER(ExpmInfo)]),
    "tns_zexpmv_gradient": (_I, [_P, _I, _I, _D, _P, _I, _P, _I, _P, _I, C.POINTER(_D), _P, _I, _P, _I,
                                 C.POINTER(_D), _P, _I, C.POINTER(ExpmInfo)]),
    "tns_set_checkpoint_bytes": (_I, [_P, _LL]),
    "tns_set_autotune": (_I, [_P, _I]),
    "tns_dnormest1_operator": (_I, [_P, _I, APPLY_FN, APPLY_FN, _P, _I, _I, _I, C.POINTER(NormestResult)]),
    "tns_znormest1_operator": (_I, [_P, _I, APPLY_FN, APPLY_FN, _P, _I, _I, _I, C.POINTER(NormestResult)]),
    "tns_dexpmv_operator": (_I, [_P, _I, APPLY_FN, _P, _I, _P, _I, _D, _D, _P, _I, C.POINTER(ExpmvInfo)]),
    "tns_zexpmv_operator": (_I, [_P, _I, APPLY_FN, _P, _I, _P, _I, _D, _D, _P, _I, C.POINTER(ExpmvInfo)]),
    "tns_dgesv_mixed": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I, _I, _I, C.POINTER(MixedInfo)]),
    "tns_zgesv_mixed": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _I, _I, _I, C.POINTER(MixedInfo)]),
    "tns_zgemm_device_noalloc": (_I, [_P, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P, _I]),
    "tns_set_workers": (_I, [_P, _I]),
    "tns_get_stats": (_I, [_P, C.POINTER(Stats)]),
    "tns_reset_stats": (_I, [_P]),
    "tns_set_timing": (_I, [_P, _I]),
    "tns_get_stream": (_I, [_P, C.POINTER(_P)]),
    "tns_set_lu_timing": (_I, [_P, _I]),
    "tns_inject_allocation_failure": (_I, [_P, _LL]),
    "tns_selftest_wait": (_I, [_P, _LL]),
    "tns_get_lu_timings": (_I, [_P, C.POINTER(LuTimings)]),
}

_lib = None


def load():
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m csharp_linearalgebra_b200.build` "
                "(nvcc, sm_100a). There is no CPU fallback.")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
