"""Row a10 against the reference's own GPU code: NumPP's CUDA backend
(src/backend/cuda_backend.cu, compiled unmodified for sm_100a into
oracle/_ref/refcuda/) computes C = A B through its GpuVTable gemm slot (host
buffers, its 16 x 16 tiled kernel); nppb_gemm (host buffers, the FP64 DMMA
kernel) must agree with it within the slot's floating-point tolerance
(gpu_vtable.hpp:22-26: accumulation order and FMA contraction differ), here
k * 2^-50 * max|A| * max|B| absolute."""
import numpy as np
import pytest

from numpp_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle.oracle import load_refcuda
    R = load_refcuda()
    if R is None:
        pytest.skip("oracle/_ref/refcuda (the reference's CUDA backend) is not built here")
    assert R.ref_cuda_available() == 1, "the reference's CUDA backend sees no device"
    return R


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (64, 48, 80), (257, 129, 300), (1000, 1024, 517), (1024, 1024, 1024)])
def test_gemm_matches_the_reference_gpu_gemm(lib, refcuda, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    Cr = np.full((m, n), np.nan)
    assert refcuda.ref_cuda_gemm(0, m, n, k, A.ctypes.data, B.ctypes.data, Cr.ctypes.data) == 1
    C = np.full((m, n), np.nan)
    assert lib.nppb_gemm(_lib.DT_FLOAT64, m, n, k, A.ctypes.data, B.ctypes.data, C.ctypes.data) == 0, _lib.last_error()
    tol = k * 2.0 ** -50 * np.abs(A).max() * np.abs(B).max()
    np.testing.assert_allclose(C, Cr, rtol=0, atol=tol)
    np.testing.assert_allclose(C, A @ B, rtol=0, atol=tol)
