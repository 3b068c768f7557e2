"""Batched Cholesky on the device against the reference's outputs (tests/golden),
the C oracle (a restatement of linalg.cpp:117-136) and numpy.

Bar: per matrix, ||L - L_oracle|| <= 1e-12 * cond(A) * ||L_oracle|| (Frobenius),
the same normwise bound the solve path is held to; the upper triangle of A is
never read; a matrix that is not positive definite fails the call."""
import ctypes as C

import numpy as np
import pytest

from numpp_b200 import _lib
from numpp_b200 import linalg as la

pytestmark = pytest.mark.gpu


def _spd(seed, cnt, n):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((cnt, n, n))
    A = X @ X.transpose(0, 2, 1) / n + np.eye(n)
    A += np.triu(rng.standard_normal((cnt, n, n)), 1)  # the upper triangle must not matter
    return A


def _close(L, Lo, A):
    sym = np.tril(A) + np.tril(A, -1).transpose(0, 2, 1)
    cond = np.linalg.cond(sym)
    err = np.linalg.norm((L - Lo).reshape(len(L), -1), axis=1)
    return np.all(err <= 1e-12 * cond * np.linalg.norm(Lo.reshape(len(L), -1), axis=1))


def test_cholesky_golden(golden, lib):
    """test_linalg.cpp:61-69, test_batched_linalg.cpp:53-58 and a seeded stack."""
    A = golden["spd3_A"]
    np.testing.assert_allclose(la.cholesky(A), golden["chol_spd3"], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(la.cholesky(golden["chol_stack_A"]), golden["chol_stack_L"], rtol=1e-14, atol=1e-15)
    L = la.cholesky(golden["chol40_A"])
    assert _close(L, golden["chol40_L"], golden["chol40_A"])
    with pytest.raises(la.LinAlgError, match=str(golden["chol_notpd_err"])):
        la.cholesky(np.array([[-1.0, 0], [0, -1]]))


@pytest.mark.parametrize("cnt,n", [(64, 1), (50, 5), (40, 16), (33, 32), (20, 33), (12, 100), (6, 300),
                                   (3, 513), (2, 1030)])
def test_cholesky_vs_oracle(oracle, lib, cnt, n):
    A = _spd(n, cnt, n)
    L = la.cholesky(A)
    Lo, ok = oracle.cholesky(A)
    assert ok.all()
    assert np.array_equal(L, np.tril(L))
    assert _close(L, Lo, A)
    sym = np.tril(A) + np.tril(A, -1).transpose(0, 2, 1)
    np.testing.assert_allclose(L @ L.transpose(0, 2, 1), sym, rtol=0, atol=1e-12 * np.abs(sym).max())


@pytest.mark.parametrize("n", [6, 40, 600])
def test_not_positive_definite(lib, n):
    A = _spd(7, 3, n)
    A[1, n // 2, n // 2] = -5.0  # system 1 fails at (or before) column n // 2
    with pytest.raises(la.LinAlgError, match="Matrix is not positive definite"):
        la.cholesky(A)
    Lm = np.empty_like(A)
    info = np.full(3, -1, np.int32)
    assert lib.nppb_cholesky_batched(3, n, _lib.ptr(A), _lib.ptr(Lm), _lib.ptr(info)) == _lib.OK
    assert info[0] == 0 and info[2] == 0 and 1 <= info[1] <= n // 2 + 1
    Lo, ok = __import__("oracle").load_oracle().cholesky(A[[0, 2]])
    assert _close(Lm[[0, 2]], Lo, A[[0, 2]])


def test_cholesky_device_entry(lib, oracle):
    import torch
    A = _spd(11, 4, 200)
    dA = torch.from_numpy(A).cuda()
    dL = torch.empty_like(dA)
    dI = torch.zeros(4, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_cholesky_batched(4, 200, C.c_void_p(dA.data_ptr()), C.c_void_p(dL.data_ptr()),
                                     C.c_void_p(dI.data_ptr()), C.c_void_p(st))
    assert rc == _lib.OK, _lib.last_error()
    torch.cuda.synchronize()
    assert not dI.any()
    Lo, _ = oracle.cholesky(A)
    assert _close(dL.cpu().numpy(), Lo, A)
    assert lib.nppb_d_cholesky_batched(1, 5000, None, None, None, None) == _lib.E_RANGE
