"""Parity of the CUDA path (through the C ABI) with the C oracle of the reference.

Tolerances (FP64 path): solutions within 1e-12 * cond(A) relative error of the
reference LU; det / slogdet within the same bound relative to their value;
pivot sequences and det signs bit-exact on tie-free seeded inputs."""
import ctypes as C

import numpy as np
import pytest

from numpp_b200 import _lib, workloads

pytestmark = pytest.mark.gpu
P = _lib.ptr


def piv_vector(ipiv):
    """LAPACK-style swap list -> the reference's permutation vector (linalg.cpp:52,60)."""
    perm = np.arange(len(ipiv))
    for k, p in enumerate(ipiv):
        perm[k], perm[p] = perm[p], perm[k]
    return perm


def rel_err(x, ref):
    x = x.reshape(x.shape[0], -1)
    ref = ref.reshape(ref.shape[0], -1)
    return np.linalg.norm(x - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)


def check_solution(x, ref, A):
    cond = np.linalg.cond(A)
    err = rel_err(x, ref)
    assert np.all(err <= 1e-12 * cond), (err / cond).max()


def gpu_solve_det(lib, A, B):
    cnt, n, k = B.shape[0], A.shape[-1], B.shape[-1]
    X = np.zeros_like(B)
    det = np.zeros(cnt)
    info = np.full(cnt, -7, np.int32)
    rc = lib.nppb_solve_det_batched(cnt, n, k, P(A), P(B), P(X), P(det), P(info))
    assert rc == 0, _lib.last_error()
    return X, det, info


def test_uniform_256x32_solve_det(lib, oracle):
    """The (256, 32, 32) + 32 I solve + det workload, seeded."""
    A, B = workloads.uniform_batch(seed=2024)
    X, det, info = gpu_solve_det(lib, A, B)
    Xo, ok = oracle.solve(A, B)
    do = oracle.det(A)
    assert ok.all() and not info.any()
    check_solution(X, Xo, A)
    assert np.array_equal(np.sign(det), np.sign(do))
    np.testing.assert_allclose(det, do, rtol=1e-12 * np.linalg.cond(A).max())


ORDERS = [1, 2, 3, 4, 5, 7, 8, 9, 12, 15, 16, 17, 24, 31, 32, 33, 40, 63, 64, 65, 96, 127, 128,
          129, 200, 255, 256, 257, 384, 511, 512]


@pytest.mark.parametrize("n", ORDERS)
def test_orders_solve_inv_det_slogdet(lib, oracle, n):
    rng = np.random.default_rng(1000 + n)
    cnt = 6
    A = rng.standard_normal((cnt, n, n))
    for k in (1, 3, 32):
        B = rng.standard_normal((cnt, n, k))
        X = np.zeros_like(B)
        info = np.zeros(cnt, np.int32)
        assert lib.nppb_solve_batched(cnt, n, k, P(A), P(B), P(X), P(info)) == 0, _lib.last_error()
        Xo, ok = oracle.solve(A, B)
        assert ok.all() and not info.any()
        check_solution(X, Xo, A)
    Ainv = np.zeros_like(A)
    info = np.zeros(cnt, np.int32)
    assert lib.nppb_inv_batched(cnt, n, P(A), P(Ainv), P(info)) == 0, _lib.last_error()
    check_solution(Ainv, oracle.inv(A)[0], A)
    det = np.zeros(cnt)
    assert lib.nppb_det_batched(cnt, n, P(A), P(det)) == 0
    do = oracle.det(A)
    assert np.array_equal(np.sign(det), np.sign(do))
    fin = np.isfinite(do) & (do != 0)
    np.testing.assert_allclose(det[fin], do[fin], rtol=1e-12 * np.linalg.cond(A).max())
    s = np.zeros(cnt)
    l = np.zeros(cnt)
    assert lib.nppb_slogdet_batched(cnt, n, P(A), P(s), P(l)) == 0
    so, lo = oracle.slogdet(A)
    assert np.array_equal(s, so)
    np.testing.assert_allclose(l, lo, rtol=1e-12 * np.linalg.cond(A).max(), atol=1e-12 * n)


@pytest.mark.parametrize("n", [5, 16, 32, 48, 64, 100, 160, 256, 400, 512])
def test_pivots_bit_exact(lib, oracle, n):
    rng = np.random.default_rng(77 + n)
    cnt = 8
    A = rng.standard_normal((cnt, n, n))
    LU = A.copy()
    ipiv = np.zeros((cnt, n), np.int32)
    info = np.zeros(cnt, np.int32)
    assert lib.nppb_getrf_batched(cnt, n, P(LU), P(ipiv), P(info)) == 0, _lib.last_error()
    assert not info.any()
    LUo, pivo, sgno, ok = oracle.lu(A)
    for i in range(cnt):
        assert np.array_equal(piv_vector(ipiv[i]), pivo[i]), f"system {i}"
        nswap = np.count_nonzero(ipiv[i] != np.arange(n))
        assert (-1.0) ** nswap == sgno[i]
    scale = np.abs(LUo).max(axis=(1, 2), keepdims=True)
    assert np.all(np.abs(LU - LUo) <= 1e-11 * np.linalg.cond(A)[:, None, None] * scale)


@pytest.mark.parametrize("n", [4, 32, 100, 512])
def test_getrs_reuses_factors(lib, oracle, n):
    rng = np.random.default_rng(5 + n)
    cnt = 4
    A = rng.standard_normal((cnt, n, n)) + n * np.eye(n)
    LU = A.copy()
    ipiv = np.zeros((cnt, n), np.int32)
    info = np.zeros(cnt, np.int32)
    assert lib.nppb_getrf_batched(cnt, n, P(LU), P(ipiv), P(info)) == 0
    for k in (1, 7):
        B = rng.standard_normal((cnt, n, k))
        Bw = B.copy()
        assert lib.nppb_getrs_batched(cnt, n, k, P(LU), P(ipiv), P(Bw)) == 0, _lib.last_error()
        check_solution(Bw, oracle.solve(A, B)[0], A)


@pytest.mark.parametrize("n", [3, 20, 32, 50, 130])
def test_singular_systems(lib, oracle, n):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((4, n, n))
    A[1] = 0.0                      # zero matrix: first pivot is zero
    A[2, n // 3] = 0.0              # zero row: stays zero, exact zero pivot at the end
    A[3, :, n // 2] = 0.0           # zero column: exact zero pivot at that column
    det = np.zeros(4)
    assert lib.nppb_det_batched(4, n, P(A), P(det)) == 0
    do = oracle.det(A)
    assert det[1] == det[2] == det[3] == 0.0 and do[1] == do[2] == do[3] == 0.0
    assert det[0] != 0.0
    s = np.zeros(4)
    l = np.zeros(4)
    assert lib.nppb_slogdet_batched(4, n, P(A), P(s), P(l)) == 0
    assert list(s[1:]) == [0.0] * 3 and np.all(np.isneginf(l[1:]))
    X = np.zeros((4, n, 1))
    info = np.zeros(4, np.int32)
    assert lib.nppb_solve_batched(4, n, 1, P(A), P(np.ones((4, n, 1))), P(X), P(info)) == 0
    _, ok = oracle.solve(A, np.ones((4, n, 1)))
    assert info[0] == 0 and np.all(info[1:] > 0)
    assert np.array_equal(info == 0, ok == 1)
    assert info[1] == 1                # zero matrix stops at the first column
    # a duplicated row is singular only up to rounding: no exact-zero promise either side
    D = A[:1].copy()
    D[0, n - 1] = D[0, 0]
    dd = np.zeros(1)
    assert lib.nppb_det_batched(1, n, P(D), P(dd)) == 0
    scale = np.prod(np.linalg.norm(D[0], axis=1))
    assert abs(dd[0]) <= 1e-10 * scale and abs(oracle.det(D)[0]) <= 1e-10 * scale


def test_zero_order_and_empty(lib):
    det = np.full(3, 7.0)
    A = np.zeros(1)
    assert lib.nppb_det_batched(3, 0, P(A), P(det)) == 0
    assert np.array_equal(det, [1.0, 1.0, 1.0])
    assert lib.nppb_det_batched(0, 5, None, None) == 0


def test_frontend_on_device(golden):
    import numpp_b200 as nb
    x = nb.solve(golden["spd3_A"], golden["spd3_b"])
    np.testing.assert_allclose(x, golden["spd3_x"], rtol=1e-13)
    np.testing.assert_allclose(nb.inv(golden["stack_A"]), golden["stack_inv"], rtol=1e-12)
    np.testing.assert_allclose(nb.det(golden["det4d_A"]), golden["det4d_det"], atol=1e-12)
    s, l = nb.slogdet(golden["sing_A"])
    assert s == 0.0 and l == -np.inf
    with pytest.raises(nb.LinAlgError, match="Singular matrix"):
        nb.inv(np.zeros((2, 2)))
    xv = nb.solve(golden["stack_A"], golden["stack_bvec"])
    np.testing.assert_allclose(xv, golden["stack_xvec"], rtol=1e-12)
    np.testing.assert_allclose(nb.solve(golden["nodal_G"], golden["nodal_I"]), golden["nodal_v"], rtol=1e-13)
    assert nb.solve(golden["f32_A"], golden["f32_A"]).dtype == np.float32
    A, B = golden["u16_A"], golden["u16_B"]
    check_solution(nb.solve(A, B), golden["u16_x"], A)
    np.testing.assert_allclose(nb.det(A), golden["u16_det"], rtol=1e-12)


def test_vtable_slots(lib, golden):
    """numpp::gpu_vtable() through its C handle: the appended slots are wired."""
    assert lib.nppb_gpu_vtable()
