"""Mixed-precision solve (FP32 factors, FP64 refinement) against the FP64
oracle on matrices of controlled condition: A = Q1 diag(sigma) Q2^T.

Bar: normwise backward error <= tol for every system (refined, or FP64
fallback when refinement stalls); forward error within 10 * kappa * tol of
x_true (forward error <= cond * backward error); refined to tol = 1e-14 the
solution is within kappa * 1e-13 of x_true and of the FP64 reference LU's."""
import numpy as np
import pytest

from numpp_b200 import workloads
from numpp_b200.mixed import solve_mixed

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kappa", [1e2, 1e4, 1e6])
@pytest.mark.parametrize("n", [64, 200])
def test_refinement_converges(lib, oracle, n, kappa):
    A, B, Xt = workloads.conditioned_batch(seed=int(n + np.log10(kappa)), count=6, n=n, kappa=kappa, nrhs=3)
    X, rep = solve_mixed(A, B, X_true=Xt)
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 0), rep  # FP32 factors suffice up to kappa*u32 << 1
    assert np.all(rep["iters"] >= 1)
    assert np.all(rep["ferr"] <= 10 * kappa * 1e-10), rep["ferr"]
    Xo, ok = oracle.solve(A, B)
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 10 * kappa * 1e-10 + kappa * 1e-13), rel


@pytest.mark.parametrize("kappa", [1e2, 1e5])
def test_refinement_to_fp64_accuracy(lib, oracle, kappa):
    A, B, Xt = workloads.conditioned_batch(seed=int(20 + np.log10(kappa)), count=5, n=128, kappa=kappa, nrhs=2)
    X, rep = solve_mixed(A, B, X_true=Xt, tol=1e-14, max_iter=20)
    assert np.all(rep["berr"] <= 1e-14), rep["berr"]
    assert np.all(rep["fallback"] == 0), rep
    assert np.all(rep["iters"] >= 2)
    assert np.all(rep["ferr"] <= kappa * 1e-13), rep["ferr"]
    Xo, _ = oracle.solve(A, B)
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= kappa * 1e-13), rel


def test_ill_conditioned_falls_back_or_converges(lib):
    A, B, Xt = workloads.conditioned_batch(seed=8, count=4, n=96, kappa=1e10, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt)
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 1)  # kappa * u32 >> 1: refinement stalls, FP64 takes over
    assert np.all(rep["info"] == 0)


def test_no_fallback_reports_the_stall(lib):
    A, B, Xt = workloads.conditioned_batch(seed=9, count=3, n=80, kappa=1e10, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, fallback=False)
    assert np.all(rep["fallback"] == 0)
    assert np.all(rep["berr"] > 1e-10)  # the stall is visible in the report


def test_badly_scaled_rows_need_equilibration(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=10, count=8, n=128, kappa=1e3, nrhs=4, row_scale_decades=6)
    X, rep = solve_mixed(A, B, X_true=Xt)
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 0), rep["fallback"]
    Xo, _ = oracle.solve(A, B)
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 1e-6), rel


def test_small_orders_take_the_fp64_kernel(lib, oracle):
    A, B = workloads.uniform_batch(seed=4, count=16, n=24, nrhs=2)
    X, rep = solve_mixed(A, B)
    assert np.all(rep["fallback"] == 1) and np.all(rep["berr"] <= 1e-14)
    Xo, _ = oracle.solve(A, B)
    np.testing.assert_allclose(X, Xo, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("factor,kappa", [("tf32", 1e2), ("tf32", 1e3), ("bf16", 1e1), ("fp32", 1e4)])
def test_tensor_core_factors_refine(lib, oracle, factor, kappa):
    """TF32 / BF16 trailing products: rougher factors, more corrections, same bar."""
    A, B, Xt = workloads.conditioned_batch(seed=40 + int(np.log10(kappa)), count=6, n=256, kappa=kappa, nrhs=4)
    X, rep = solve_mixed(A, B, X_true=Xt, factor=factor, max_iter=30)
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 0), rep
    Xo, _ = oracle.solve(A, B)
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 10 * kappa * 1e-10 + kappa * 1e-13), rel


def test_bf16_factors_fall_back_when_too_rough(lib):
    """kappa * u_bf16 >> 1: refinement cannot contract; every system still meets the bar via FP64."""
    A, B, Xt = workloads.conditioned_batch(seed=44, count=4, n=128, kappa=1e6, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, factor="bf16")
    assert np.all(rep["berr"] <= 1e-10), rep["berr"]
    assert np.all(rep["fallback"] == 1)


@pytest.mark.parametrize("factor", ["3xtf32", "tf32"])
@pytest.mark.parametrize("n", [96, 301, 1030])
def test_tcgen05_update_matches_mma_sync(lib, factor, n):
    """The tcgen05 (TMEM accumulator) trailing update and the mma.sync one give
    factors of the same quality: same corrections, no fallback, close solutions.
    n = 301 takes the 4-byte staging path (rows not 16-byte aligned), 1030 several
    128-row tiles and 512-row groups."""
    kappa = 1e2 if factor == "tf32" else 1e4
    A, B, Xt = workloads.conditioned_batch(seed=60 + n, count=3, n=n, kappa=kappa, nrhs=2)
    Xa, ra = solve_mixed(A, B, X_true=Xt, factor=factor, max_iter=30, tcgen05=True)
    Xb, rb = solve_mixed(A, B, X_true=Xt, factor=factor, max_iter=30, pivoted=True)
    for rep in (ra, rb):
        assert np.all(rep["berr"] <= 1e-10), rep["berr"]
        assert np.all(rep["fallback"] == 0), rep
    assert np.all(np.abs(ra["iters"] - rb["iters"]) <= 1), (ra["iters"], rb["iters"])
    rel = np.abs(Xa - Xb).max(axis=(1, 2)) / np.abs(Xb).max(axis=(1, 2))
    assert np.all(rel <= 10 * kappa * 1e-10), rel
