"""The C-ABI library loads, exports every symbol include/numpp_b200*.h declare,
and fails loudly (an error status, no fallback) where no sm_100 device is visible.
No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from numpp_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("numpp_b200.h", "numpp_b200_dlpack.h")]


def declared():
    text = "".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nppb_\w+)\s*\(", text)))


def test_header_declares_the_path():
    names = declared()
    for must in ("nppb_gemm", "nppb_solve_batched", "nppb_inv_batched", "nppb_det_batched",
                 "nppb_slogdet_batched", "nppb_getrf_batched", "nppb_getrs_batched",
                 "nppb_plan_create", "nppb_plan_execute", "nppb_dl_linalg", "nppb_dl_matmul",
                 "nppb_dl_cholesky", "nppb_cholesky_batched"):
        assert must in names


def test_every_declared_symbol_is_exported():
    L = _lib.load()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding knows every one of them
    assert set(declared()) <= set(_lib.SIGNATURES), set(declared()) - set(_lib.SIGNATURES)


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    syms = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for n in declared():
        assert n in syms, n  # unmangled


def test_library_reports_version_and_no_device_here():
    L = _lib.load()
    assert L.nppb_abi_version() == 1
    assert L.nppb_max_order() >= 512
    if L.nppb_device_available():
        pytest.skip("a GPU is visible; the no-device path is not reachable")
    assert L.nppb_gpu_vtable() is None
    A = np.eye(3)[None].copy()
    X = np.zeros((1, 3, 1))
    info = np.zeros(1, np.int32)
    rc = L.nppb_solve_batched(1, 3, 1, A.ctypes.data, X.ctypes.data, X.ctypes.data, info.ctypes.data)
    assert rc == _lib.E_NODEV
    assert _lib.last_error()


def test_argument_errors_before_device_work():
    L = _lib.load()
    assert L.nppb_solve_batched(-1, 3, 1, None, None, None, None) == _lib.E_ARG
    assert L.nppb_solve_batched(1, 100000, 1, None, None, None, None) == _lib.E_RANGE
    assert L.nppb_elementwise_binary(0, 11, 4, None, None, None) == _lib.DECLINED
    assert L.nppb_gemm(5, 2, 2, 2, None, None, None) == _lib.DECLINED  # int64 gemm: CPU path
    h = C.c_void_p()
    assert L.nppb_plan_create(C.byref(h), -3, None, None, None, None, None, 2) == _lib.E_ARG


def test_argument_errors_before_any_device_work():
    """Bad sizes are refused with an error status and a message, whether or
    not a device is present (the checks come before the device probe)."""
    L = _lib.load()
    z = np.zeros(4)
    cases = [
        (L.nppb_gemm_batched, (-1, 2, 2, 2, z.ctypes.data, z.ctypes.data, z.ctypes.data), _lib.E_ARG),
        (L.nppb_d_gemm_batched, (1, -2, 2, 2, None, None, None, None), _lib.E_ARG),
        (L.nppb_matrix_power_batched, (-1, 2, 3, z.ctypes.data, z.ctypes.data, None), _lib.E_ARG),
        (L.nppb_cholesky_batched, (1, 5000, z.ctypes.data, z.ctypes.data, z.ctypes.data), _lib.E_RANGE),
        (L.nppb_d_cholesky_batched, (-3, 4, None, None, None, None), _lib.E_ARG),
        (L.nppb_solve_batched, (1, 5000, 1, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data),
         _lib.E_RANGE),
    ]
    for fn, args, want in cases:
        assert fn(*args) == want, fn.__name__
        assert _lib.last_error()
    # nothing to do is not an error
    assert L.nppb_cholesky_batched(0, 4, None, None, None) == _lib.OK
    assert L.nppb_gemm_batched(0, 2, 2, 2, None, None, None) == _lib.OK
