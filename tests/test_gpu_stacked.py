"""Stacked matmul, matrix_power, tensorsolve / tensorinv and cond on the device,
against the reference's own outputs (tests/golden) and numpy.

Tolerance: for a power p the relative max-abs error is bounded by
1e-12 * max(1, |p|) * cond(A)^(p < 0) -- every product adds one rounding of
the FP64 GEMM, and a negative power starts from an inverse within 1e-12 * cond(A).
The batched GEMM is within 1e-13 relative to |A| |B| (k-term FP64 dot products)."""
import ctypes as C

import numpy as np
import pytest

from numpp_b200 import _lib
from numpp_b200 import linalg as la

pytestmark = pytest.mark.gpu


def _gemm_bound(A, B):
    return np.abs(A) @ np.abs(B)


def _power_ok(R, G, A, p):
    kappa = np.linalg.cond(A) if p < 0 else np.ones(A.shape[:-2])
    scale = np.abs(G).max(axis=(-2, -1))
    err = np.abs(R - G).max(axis=(-2, -1)) / scale
    return np.all(err <= 1e-12 * max(1, abs(p)) * kappa), err.max()


@pytest.mark.parametrize("cnt,m,k,n", [(1, 1, 1, 1), (3, 5, 7, 9), (700, 4, 4, 4), (2, 130, 67, 129),
                                       (5, 64, 0, 32), (70000, 2, 3, 2)])
def test_gemm_batched_host(lib, cnt, m, k, n):
    rng = np.random.default_rng(cnt + m + k + n)
    A = rng.standard_normal((cnt, m, k))
    B = rng.standard_normal((cnt, k, n))
    Cm = la.matmul_batched(A, B)
    assert Cm.shape == (cnt, m, n)
    ref = np.einsum("zmk,zkn->zmn", A, B)
    assert np.all(np.abs(Cm - ref) <= 1e-13 * (_gemm_bound(A, B) + 1e-300))


def test_gemm_batched_broadcast_and_dtype(lib):
    rng = np.random.default_rng(11)
    A = rng.standard_normal((4, 1, 6, 5))
    B = rng.standard_normal((3, 5, 7))
    np.testing.assert_allclose(la.matmul_batched(A, B), A @ B, rtol=1e-13, atol=1e-13)
    Cf = la.matmul_batched(A.astype(np.float32), B.astype(np.float32))
    assert Cf.dtype == np.float32
    np.testing.assert_allclose(Cf, (A.astype(np.float32) @ B.astype(np.float32)), rtol=1e-5, atol=1e-5)


def test_gemm_batched_device_entry(lib):
    import torch
    rng = np.random.default_rng(12)
    A = rng.standard_normal((9, 33, 17))
    B = rng.standard_normal((9, 17, 65))
    dA = torch.from_numpy(A).cuda()
    dB = torch.from_numpy(B).cuda()
    dC = torch.empty((9, 33, 65), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_gemm_batched(9, 33, 65, 17, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                 C.c_void_p(dC.data_ptr()), C.c_void_p(st))
    assert rc == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    assert np.all(np.abs(dC.cpu().numpy() - A @ B) <= 1e-13 * _gemm_bound(A, B))
    assert lib.nppb_d_gemm_batched(-1, 2, 2, 2, None, None, None, None) == _lib.E_ARG


def test_matrix_power_golden(golden, lib):
    """test_linalg_mined3.cpp:29-40 and the seeded (6, 9, 9) stack."""
    P = golden["mp2_A"]
    for p in (0, 1, 2, 7, -1, -3):
        R = la.matrix_power(P, p)
        ok, err = _power_ok(R, golden[f"mp2_p{p}"], P, p)
        assert ok, (p, err)
    assert np.array_equal(la.matrix_power(P, 0), np.eye(2))
    assert np.array_equal(la.matrix_power(P, 1), P)
    assert la.matrix_power(P.astype(np.float32), 0).dtype == golden["mp2_f32_p0"].dtype
    for p in (3, 8, -2, -4):
        ok, err = _power_ok(la.matrix_power(golden["mp9_A"], p), golden[f"mp9_p{p}"], golden["mp9_A"], p)
        assert ok, (p, err)
    with pytest.raises(la.LinAlgError, match=str(golden["mp_sing_err"])):
        la.matrix_power(golden["sing_A"], -1)


@pytest.mark.parametrize("shape,p", [((64, 64, 64), 5), ((64, 64, 64), -3), ((2, 300, 300), 2),
                                     ((4, 3, 130, 130), 13), ((1000, 8, 8), -6)])
def test_matrix_power_vs_numpy(lib, shape, p):
    n = shape[-1]
    rng = np.random.default_rng(n + abs(p))
    A = rng.standard_normal(shape) / np.sqrt(n) + 0.6 * np.eye(n)
    R = la.matrix_power(A, p)
    ok, err = _power_ok(R, np.linalg.matrix_power(A, p), A, p)
    assert ok, err


def test_matrix_power_singular_in_stack(lib):
    A = np.stack([np.eye(5) * 2.0, np.zeros((5, 5)), np.eye(5)])
    with pytest.raises(la.LinAlgError, match="Singular matrix"):
        la.matrix_power(A, -2)
    R = la.matrix_power(A, 3)   # positive powers never invert
    assert np.array_equal(R[0], np.eye(5) * 8.0) and np.array_equal(R[1], np.zeros((5, 5)))


def test_matrix_power_abi_info(lib):
    A = np.stack([np.eye(4) * 2.0, np.zeros((4, 4))])
    R = np.empty_like(A)
    info = np.full(2, -7, np.int32)
    assert lib.nppb_matrix_power_batched(2, 4, -1, _lib.ptr(A), _lib.ptr(R), _lib.ptr(info)) == _lib.OK
    assert info[0] == 0 and info[1] != 0
    np.testing.assert_array_equal(R[0], np.eye(4) * 0.5)


def test_tensorsolve_tensorinv_golden(golden, lib):
    """tensor_solve.cpp:10-49 on the device against the reference's outputs."""
    T, b = golden["tens_A"], golden["tens_b"]
    np.testing.assert_allclose(la.tensorsolve(T, b), golden["tens_x"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(la.tensorsolve(T, b, axes=(0,)), golden["tens_x_ax0"], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(la.tensorinv(T, 2), golden["tens_inv"], rtol=1e-13, atol=1e-15)
    A3 = golden["tens3_A"]
    k3 = np.linalg.cond(A3.reshape(12, 12))
    x3 = la.tensorsolve(A3, golden["tens3_b"])
    assert np.abs(x3 - golden["tens3_x"]).max() <= 1e-12 * k3 * np.abs(golden["tens3_x"]).max()
    A4 = golden["tens4_A"]
    k4 = np.linalg.cond(A4.reshape(24, 24))
    t4 = la.tensorinv(A4, 2)
    assert t4.shape == (8, 3, 4, 6)
    assert np.abs(t4 - golden["tens4_inv"]).max() <= 1e-12 * k4 * np.abs(golden["tens4_inv"]).max()


def test_cond(lib):
    rng = np.random.default_rng(21)
    A = rng.standard_normal((5, 40, 40)) + 5 * np.eye(40)
    for p in (1, -1, np.inf, -np.inf, "fro"):
        np.testing.assert_allclose(la.cond(A, p), np.linalg.cond(A, p), rtol=1e-11)
    S = np.stack([A[0], np.zeros((40, 40))])
    c = la.cond(S, np.inf)
    assert np.isfinite(c[0]) and c[1] == np.inf
