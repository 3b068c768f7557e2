"""ctypes binding of libnumpp_b200.so (the C ABI declared in include/numpp_b200.h
and include/numpp_b200_dlpack.h).

Loading fails loudly: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnumpp_b200.so")

# status codes (numpp_b200.h)
OK, DECLINED = 0, 1
E_ARG, E_NODEV, E_CUDA, E_NOMEM, E_RANGE = -1, -2, -3, -4, -5
DT_FLOAT32, DT_FLOAT64 = 10, 11
WANT_LU, WANT_SOLVE, WANT_DET, WANT_SLOGDET, WANT_INV = 1, 2, 4, 8, 16
MIXED_NO_EQUILIBRATE, MIXED_NO_FALLBACK, MIXED_TF32, MIXED_BF16, MIXED_FP32_FMA, MIXED_TCGEN05 = 1, 2, 4, 8, 16, 32
MIXED_PIVOTED = 64
MIXED_GMRES = 128

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_int = C.c_int

# name -> (restype, argtypes); every symbol include/numpp_b200*.h declare.
SIGNATURES = {
    "nppb_abi_version": (_int, []),
    "nppb_device_available": (_int, []),
    "nppb_last_error": (C.c_char_p, []),
    "nppb_max_order": (_i32, []),
    "nppb_gpu_vtable": (_vp, []),
    "nppb_elementwise_binary": (_int, [_int, _int, _i64, _vp, _vp, _vp]),
    "nppb_elementwise_unary": (_int, [_int, _int, _i64, _vp, _vp]),
    "nppb_reduce": (_int, [_int, _int, _i64, _vp, _vp]),
    "nppb_gemm": (_int, [_int, _i64, _i64, _i64, _vp, _vp, _vp]),
    "nppb_d_gemm": (_int, [_int, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
    "nppb_getrf_batched": (_int, [_i64, _i32, _vp, _vp, _vp]),
    "nppb_getrs_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp]),
    "nppb_solve_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp]),
    "nppb_inv_batched": (_int, [_i64, _i32, _vp, _vp, _vp]),
    "nppb_det_batched": (_int, [_i64, _i32, _vp, _vp]),
    "nppb_slogdet_batched": (_int, [_i64, _i32, _vp, _vp, _vp]),
    "nppb_solve_det_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "nppb_d_linalg_batched": (_int, [_i64, _i32, _i32, _int] + [_vp] * 10 + [_vp]),
    "nppb_d_getrs_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "nppb_d_solve_batched_noalloc": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "nppb_d_solve_mixed_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp, C.c_double, _i32, _int,
                                          _vp, _vp, _vp, _vp, _vp, _vp]),
    "nppb_solve_mixed_batched": (_int, [_i64, _i32, _i32, _vp, _vp, _vp, _vp, C.c_double, _i32, _int,
                                        _vp, _vp, _vp, _vp, _vp]),
    "nppb_plan_create": (_int, [C.POINTER(_vp), _i64, _vp, _vp, _vp, _vp, _vp, _int]),
    "nppb_plan_sizes": (_int, [_vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "nppb_plan_execute": (_int, [_vp] * 10),
    "nppb_plan_execute_host": (_int, [_vp] * 9),
    "nppb_plan_destroy": (_int, [_vp]),
    "nppb_plan_num_classes": (_int, [_vp]),
    "nppb_plan_num_launches": (_int, [_vp]),
    "nppb_plan_class_info": (_int, [_vp, _int, C.POINTER(_int), C.POINTER(_int), C.POINTER(_i64),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nppb_plan_time_classes": (_int, [_vp] * 10 + [_int, C.POINTER(C.c_float)]),
    "nppb_plan_autotune": (_int, [_vp] * 10 + [C.POINTER(_i32), C.POINTER(C.c_float)]),
    "nppb_autotune_key": (_int, [C.c_int64, _vp, _vp, C.c_int, C.c_char_p, C.c_int64]),
    "nppb_autotune_cache_get": (_int, [C.c_char_p, C.POINTER(_i32), C.POINTER(C.c_float), C.POINTER(_i32)]),
    "nppb_autotune_cache_put": (_int, [C.c_char_p, _i32, C.c_float]),
    "nppb_plan_time_kernels": (_int, [_vp] * 10 + [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nppb_solve_grouped": (_int, [_i64, _vp, _vp, _vp, _vp, _vp, _int] + [_vp] * 8),
    "nppb_d_gemm_batched": (_int, [_i64, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
    "nppb_gemm_batched": (_int, [_i64, _i64, _i64, _i64, _vp, _vp, _vp]),
    "nppb_matrix_power_batched": (_int, [_i64, _i32, _i64, _vp, _vp, _vp]),
    "nppb_cholesky_batched": (_int, [_i64, _i32, _vp, _vp, _vp]),
    "nppb_d_cholesky_batched": (_int, [_i64, _i32, _vp, _vp, _vp, _vp]),
    "nppb_lstsq_batched": (_int, [_i64, _i32, _i32, _i32, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp, _vp]),
    "nppb_d_lstsq_batched": (_int, [_i64, _i32, _i32, _i32, _vp, _vp, C.c_double, _vp, _vp, _vp, _vp, _vp, _vp]),
    "nppb_dl_linalg": (_int, [_int] + [_vp] * 9),
    "nppb_dl_matmul": (_int, [_vp] * 4),
    "nppb_dl_cholesky": (_int, [_vp] * 4),
    "nppb_server_create": (_int, [C.POINTER(_vp), _i64, C.c_double, _i32]),
    "nppb_server_submit": (_int, [_vp, _i32, _i32, _vp, _vp, _vp, _i64, _i32, C.POINTER(_i64), C.POINTER(_i64)]),
    "nppb_server_wait": (_int, [_vp, _i64, C.c_double, C.POINTER(_i32), C.POINTER(C.c_double)]),
    "nppb_server_release_factor": (_int, [_vp, _i64]),
    "nppb_server_stats": (_int, [_vp, C.POINTER(_i64)]),
    "nppb_server_destroy": (_int, [_vp]),
}

_LIB = None


class NativeMissing(ImportError):
    pass


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load the library once and bind every declared entry point."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise NativeMissing(
            f"{path} is missing: build it with numpp_b200.build.build() "
            "(the B200 path has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def last_error() -> str:
    msg = load().nppb_last_error()
    return msg.decode() if msg else ""


def ptr(a) -> int | None:
    """Address of a numpy array / torch tensor / int / None for a void* argument."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
