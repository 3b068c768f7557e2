"""GpuVTable::gemm on DMMA vs the reference's CPU GEMM (tests/test_gpu.cpp:56-79:
allclose 1e-10 / 1e-10)."""
import numpy as np
import pytest

from numpp_b200 import _lib

pytestmark = pytest.mark.gpu
P = _lib.ptr


def gemm(lib, A, B, dt=_lib.DT_FLOAT64):
    m, k = A.shape
    n = B.shape[1]
    C = np.zeros((m, n), A.dtype)
    assert lib.nppb_gemm(dt, m, n, k, P(A), P(B), P(C)) == 0, _lib.last_error()
    return C


def test_reference_case(lib, golden):
    C = gemm(lib, golden["gemm_A"], golden["gemm_B"])
    np.testing.assert_allclose(C, golden["gemm_C"], rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (129, 65, 33), (128, 64, 8), (300, 517, 1001),
                                   (1024, 1024, 1024), (5, 3, 0)])
def test_shapes_vs_oracle(lib, oracle, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C = gemm(lib, A, B)
    Co = oracle.matmul(A, B) if k else np.zeros((m, n))
    tol = 1e-14 * max(k, 1) * np.abs(A).max(initial=1) * np.abs(B).max(initial=1)
    assert np.abs(C - Co).max(initial=0) <= tol


def test_float32(lib):
    rng = np.random.default_rng(1)
    A = rng.standard_normal((100, 70)).astype(np.float32)
    B = rng.standard_normal((70, 90)).astype(np.float32)
    C = gemm(lib, A, B, _lib.DT_FLOAT32)
    np.testing.assert_allclose(C, A.astype(np.float64) @ B, rtol=1e-4, atol=1e-4)
