"""Orders 513..4096: the cluster panel (2, 4 or 8 CTAs per system) and the
windowed substitutions, against the C oracle of the reference.

Same bar as the smaller orders: solutions within 1e-12 * cond(A) of the
reference LU, pivot sequences and det signs bit-exact on tie-free seeded
inputs, log|det| within 1e-12 * cond(A)."""
import numpy as np
import pytest

from numpp_b200 import _lib, workloads
from numpp_b200.grouped import solve_grouped
from numpp_b200.mixed import solve_mixed

from test_gpu_parity import check_solution, piv_vector

pytestmark = pytest.mark.gpu
P = _lib.ptr


@pytest.mark.parametrize("n,cnt", [(513, 3), (700, 2), (1024, 2), (1025, 1), (1500, 1), (2049, 1)])
def test_large_orders_solve_slogdet(lib, oracle, n, cnt):
    rng = np.random.default_rng(3000 + n)
    A = rng.standard_normal((cnt, n, n))
    for k in (1, 33):
        B = rng.standard_normal((cnt, n, k))
        X = np.zeros_like(B)
        info = np.full(cnt, -1, np.int32)
        assert lib.nppb_solve_batched(cnt, n, k, P(A), P(B), P(X), P(info)) == 0, _lib.last_error()
        Xo, ok = oracle.solve(A, B)
        assert ok.all() and not info.any()
        check_solution(X, Xo, A)
    s = np.zeros(cnt)
    l = np.zeros(cnt)
    assert lib.nppb_slogdet_batched(cnt, n, P(A), P(s), P(l)) == 0
    so, lo = oracle.slogdet(A)
    assert np.array_equal(s, so)
    np.testing.assert_allclose(l, lo, rtol=1e-12 * np.linalg.cond(A).max(), atol=1e-12 * n)


@pytest.mark.parametrize("n", [600, 1100, 2100, 4096])
def test_large_pivots_bit_exact(lib, oracle, n):
    rng = np.random.default_rng(91 + n)
    A = rng.standard_normal((1, n, n))
    LU = A.copy()
    ipiv = np.zeros((1, n), np.int32)
    info = np.zeros(1, np.int32)
    assert lib.nppb_getrf_batched(1, n, P(LU), P(ipiv), P(info)) == 0, _lib.last_error()
    assert not info.any()
    LUo, pivo, sgno, ok = oracle.lu(A)
    assert np.array_equal(piv_vector(ipiv[0]), pivo[0])
    nswap = np.count_nonzero(ipiv[0] != np.arange(n))
    assert (-1.0) ** nswap == sgno[0]
    # factors: entrywise against the reference's, scaled by the growth of U
    assert np.abs(LU - LUo).max() <= 1e-12 * n * np.abs(LUo).max()


@pytest.mark.parametrize("n", [700, 1300])
def test_large_getrs_windows(lib, oracle, n):
    rng = np.random.default_rng(17 + n)
    A = rng.standard_normal((2, n, n)) + np.sqrt(n) * np.eye(n)
    LU = A.copy()
    ipiv = np.zeros((2, n), np.int32)
    info = np.zeros(2, np.int32)
    assert lib.nppb_getrf_batched(2, n, P(LU), P(ipiv), P(info)) == 0
    for k in (1, 5, 70):
        B = rng.standard_normal((2, n, k))
        Bw = B.copy()
        assert lib.nppb_getrs_batched(2, n, k, P(LU), P(ipiv), P(Bw)) == 0, _lib.last_error()
        check_solution(Bw, oracle.solve(A, B)[0], A)


def test_large_inverse(lib, oracle):
    n = 600
    A = np.random.default_rng(5).standard_normal((2, n, n))
    Ainv = np.zeros_like(A)
    info = np.zeros(2, np.int32)
    assert lib.nppb_inv_batched(2, n, P(A), P(Ainv), P(info)) == 0, _lib.last_error()
    check_solution(Ainv, oracle.inv(A)[0], A)


def test_uneven_plan_with_large_orders(lib, oracle):
    """One plan over orders that take every panel class, warp kernel included."""
    sys = workloads.packed_batch(31, n=[33, 300, 513, 777, 1030, 64, 2050, 20, 520, 1500, 8, 129],
                                 nrhs=[1, 8, 32, 1, 8, 32, 1, 8, 32, 1, 8, 32],
                                 want_inv=[0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0])
    X, Inv, Det, Sign, Logabs, info = solve_grouped(sys)
    Xo, so, lo, invo, ok = oracle.solve_grouped(sys)
    assert ok.all() and not info.any()
    for i in range(len(sys["n"])):
        n, k = int(sys["n"][i]), int(sys["nrhs"][i])
        A = sys["A"][sys["a_off"][i]:sys["a_off"][i] + n * n].reshape(1, n, n)
        xb = slice(sys["b_off"][i], sys["b_off"][i] + n * k)
        check_solution(X[xb].reshape(1, n, k), Xo[xb].reshape(1, n, k), A)
        cond = np.linalg.cond(A[0])
        assert Sign[i] == so[i], i
        assert abs(Logabs[i] - lo[i]) <= 1e-12 * cond * max(1.0, abs(lo[i])), i
        if sys["inv_off"][i] >= 0:
            ib = slice(sys["inv_off"][i], sys["inv_off"][i] + n * n)
            check_solution(Inv[ib].reshape(1, n, n), invo[ib].reshape(1, n, n), A)


@pytest.mark.parametrize("n,cnt,kappa", [(1024, 2, 1e4), (2048, 1, 1e6)])
def test_mixed_large_orders(lib, n, cnt, kappa):
    A, B, Xt = workloads.conditioned_batch(seed=n, count=cnt, n=n, kappa=kappa, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt)
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 0), rep
    assert np.all(rep["ferr"] <= 10 * kappa * 1e-10), rep["ferr"]
