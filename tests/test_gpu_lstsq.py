"""lstsq, svdvals and the 2-norm cond on the device against the reference's
outputs (tests/golden, from its Jacobi-SVD lstsq) and numpy.

Bars: singular values within 1e-13 * s_max; rank exact; the solution within
1e-12 * cond(A) relative to its norm (cond over the kept singular values);
residuals within 1e-10 relative (they are differences of nearly equal
quantities only when the fit is nearly exact, and then they are tiny)."""
import ctypes as C

import numpy as np
import pytest

from numpp_b200 import _lib
from numpp_b200 import linalg as la

pytestmark = pytest.mark.gpu

KEYS = ("R", "W", "tall", "wide", "sq", "def")


def _check(A, b, x, res, rk, sv, xo, reso, rko, svo):
    assert rk == rko
    np.testing.assert_allclose(sv, svo, rtol=0, atol=1e-13 * svo[0])
    kept = svo[svo > svo[0] * 2.220446049250313e-16 * max(A.shape)]
    cond = kept[0] / kept[-1]
    assert np.linalg.norm(x - xo) <= 1e-12 * cond * max(np.linalg.norm(xo), 1e-300)
    assert res.shape == reso.shape
    if reso.size:
        np.testing.assert_allclose(res, reso, rtol=1e-10, atol=1e-12 * np.abs(b).max() ** 2)


def test_lstsq_golden(golden, lib):
    for key in KEYS:
        A, b = golden[f"lsq_{key}_A"], golden[f"lsq_{key}_b"]
        x, res, rk, sv = la.lstsq(A, b)
        _check(A, b, x, res, rk, sv, golden[f"lsq_{key}_x"], golden[f"lsq_{key}_res"],
               int(golden[f"lsq_{key}_rank"]), golden[f"lsq_{key}_s"])


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (5, 3, 1), (3, 5, 2), (200, 64, 4), (64, 200, 3), (512, 32, 8),
                                   (3000, 8, 2), (40, 40, 5)])
def test_lstsq_vs_oracle(oracle, lib, m, n, k):
    rng = np.random.default_rng(m * 7 + n)
    A = rng.standard_normal((m, n))
    b = rng.standard_normal((m, k))
    x, res, rk, sv = la.lstsq(A, b)
    xo, reso, rko, svo = oracle.lstsq(A, b)
    _check(A, b, x, res, rk, sv, xo, reso, rko, svo)
    xn = np.linalg.lstsq(A, b, rcond=None)[0]
    np.testing.assert_allclose(x, xn, rtol=1e-9, atol=1e-10 * np.abs(xn).max())


def test_rank_deficient_minimum_norm(lib, oracle):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((30, 5)) @ rng.standard_normal((5, 12))  # rank 5
    b = rng.standard_normal(30)
    x, res, rk, sv = la.lstsq(A, b)
    xo, reso, rko, svo = oracle.lstsq(A, b)
    assert rk == rko == 5 and res.size == 0
    np.testing.assert_allclose(x, np.linalg.pinv(A) @ b, rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(x, xo, rtol=1e-8, atol=1e-10)


def test_svdvals_and_cond(lib):
    rng = np.random.default_rng(4)
    A = rng.standard_normal((6, 2, 50, 30))
    np.testing.assert_allclose(la.svdvals(A), np.linalg.svd(A, compute_uv=False), rtol=1e-12, atol=1e-13)
    S = rng.standard_normal((4, 20, 20)) + 3 * np.eye(20)
    for p in (None, 2, -2):
        np.testing.assert_allclose(la.cond(S, p), np.linalg.cond(S, p), rtol=1e-11)
    assert la.cond(np.zeros((3, 3))) == np.inf and la.cond(np.zeros((3, 3)), -2) == 0.0


def test_declined_and_device_entry(lib):
    import torch
    with pytest.raises(la.Declined):
        la.lstsq(np.ones((100, 100)), np.ones(100))      # min(m, n) = 100 > 64
    rng = np.random.default_rng(5)
    A = rng.standard_normal((7, 40, 10))
    B = rng.standard_normal((7, 40, 2))
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    dX = torch.empty(7, 10, 2, dtype=torch.float64, device="cuda")
    dS = torch.empty(7, 10, dtype=torch.float64, device="cuda")
    dR = torch.empty(7, dtype=torch.int32, device="cuda")
    dres = torch.empty(7, 2, dtype=torch.float64, device="cuda")
    dh = torch.empty(7, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_lstsq_batched(7, 40, 10, 2, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()), -1.0,
                                  C.c_void_p(dX.data_ptr()), C.c_void_p(dS.data_ptr()), C.c_void_p(dR.data_ptr()),
                                  C.c_void_p(dres.data_ptr()), C.c_void_p(dh.data_ptr()), C.c_void_p(st))
    assert rc == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    assert bool((dR == 10).all()) and bool((dh == 1).all())
    for i in range(7):
        xn, rn = np.linalg.lstsq(A[i], B[i], rcond=None)[:2]
        np.testing.assert_allclose(dX[i].cpu().numpy(), xn, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(dres[i].cpu().numpy(), rn, rtol=1e-10)


def test_rcond_and_wide_rank_deficient(lib, oracle):
    """An explicit rcond drops the same singular values as the reference; a
    wide rank-deficient problem gives the minimum-norm solution."""
    rng = np.random.default_rng(8)
    A = rng.standard_normal((25, 12)) @ np.diag(np.logspace(0, -9, 12)) @ rng.standard_normal((12, 12))
    b = rng.standard_normal((25, 2))
    for rcond in (1e-4, 1e-7, 0.0):
        x, res, rk, sv = la.lstsq(A, b, rcond=rcond)
        xo, reso, rko, svo = oracle.lstsq(A, b, rcond)
        assert rk == rko, rcond
        np.testing.assert_allclose(sv, svo, rtol=0, atol=1e-13 * svo[0])
        if rk < 12:
            np.testing.assert_allclose(x, xo, rtol=1e-8, atol=1e-9 * np.abs(xo).max())
    W = rng.standard_normal((6, 3)) @ rng.standard_normal((3, 20))  # 6 x 20, rank 3
    bw = rng.standard_normal(6)
    x, res, rk, sv = la.lstsq(W, bw)
    assert rk == 3 and res.size == 0
    np.testing.assert_allclose(x, np.linalg.pinv(W) @ bw, rtol=1e-8, atol=1e-10)
