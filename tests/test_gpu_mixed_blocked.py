"""The mixed solve's default factorisation: random butterflies, pivoting inside
each 128-row diagonal block, triangular solves and trailing updates as
tcgen05 GEMMs (error-compensated TF32, TMEM accumulators, TMA-staged tiles),
FP64 refinement. Against the oracle (the reference's LU restated) and x_true.

Bar, as for the other mixed tests: normwise backward error <= tol for every
system; forward error <= 10 * kappa * tol; solutions within 10 * kappa * tol
(+ kappa * 1e-13) of the oracle's. Orders cover one block, padding to the
next multiple of 128 and several blocks; right-hand-side counts cover the
substitution's chunks of 1, 2, 4 and 8 columns."""
import numpy as np
import pytest

from numpp_b200 import workloads
from numpp_b200.mixed import solve_mixed

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _check(oracle, A, B, Xt, X, rep, kappa, fallback_ok=False):
    assert np.all(rep["berr"] <= TOL), rep["berr"]
    if not fallback_ok:
        assert np.all(rep["fallback"] == 0), rep
        assert np.all(rep["iters"] >= 1)
    assert np.all(rep["ferr"] <= 10 * kappa * TOL), rep["ferr"]
    Xo, ok = oracle.solve(A, B)
    assert ok.all()
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 10 * kappa * TOL + kappa * 1e-13), rel


@pytest.mark.parametrize("n", [33, 100, 128, 129, 256, 300, 640])
@pytest.mark.parametrize("kappa", [1e2, 1e4])
def test_blocked_orders(lib, oracle, n, kappa):
    A, B, Xt = workloads.conditioned_batch(seed=7 * n + int(np.log10(kappa)), count=4, n=n, kappa=kappa, nrhs=2)
    X, rep = solve_mixed(A, B, X_true=Xt)
    _check(oracle, A, B, Xt, X, rep, kappa)


@pytest.mark.parametrize("nrhs", [1, 3, 4, 9, 64])
def test_blocked_rhs_chunks(lib, oracle, nrhs):
    A, B, Xt = workloads.conditioned_batch(seed=100 + nrhs, count=3, n=384, kappa=1e3, nrhs=nrhs)
    X, rep = solve_mixed(A, B, X_true=Xt)
    _check(oracle, A, B, Xt, X, rep, 1e3)


def test_blocked_kappa_1e6(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=61, count=4, n=256, kappa=1e6, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, max_iter=30)
    _check(oracle, A, B, Xt, X, rep, 1e6, fallback_ok=True)


def test_blocked_row_scaled(lib, oracle):
    """rows scaled by 10^U(-6, 6): equilibration before the transform"""
    A, B, Xt = workloads.conditioned_batch(seed=62, count=6, n=256, kappa=1e3, nrhs=4, row_scale_decades=6)
    X, rep = solve_mixed(A, B, X_true=Xt)
    _check(oracle, A, B, Xt, X, rep, 1e3)


def test_blocked_tight_tolerance(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=63, count=3, n=256, kappa=1e2, nrhs=2)
    X, rep = solve_mixed(A, B, X_true=Xt, tol=1e-14, max_iter=20)
    assert np.all(rep["berr"] <= 1e-14) and np.all(rep["fallback"] == 0), rep
    Xo, _ = oracle.solve(A, B)
    rel = np.abs(X - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 1e2 * 1e-13), rel


def test_blocked_singular_system_falls_back(lib):
    """An exactly singular system cannot refine; the FP64 solve reports it."""
    A, B, Xt = workloads.conditioned_batch(seed=64, count=3, n=200, kappa=1e2, nrhs=1)
    A[1, 7] = 0.0
    A[1, 9] = 0.0  # two zero rows: singular
    X, rep = solve_mixed(A, B, X_true=Xt)
    assert rep["fallback"][1] == 1 and rep["info"][1] > 0
    for s in (0, 2):
        assert rep["fallback"][s] == 0 and rep["berr"][s] <= TOL


def test_blocked_no_fallback_reports_the_stall(lib):
    A, B, Xt = workloads.conditioned_batch(seed=65, count=3, n=160, kappa=1e10, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, fallback=False)
    assert np.all(rep["fallback"] == 0)
    assert np.all(rep["berr"] > TOL)


def test_blocked_alone_and_in_a_batch_agree_bitwise(lib):
    """Every kernel's arithmetic for a system depends only on that system: a
    system solved alone and inside a batch gives the same bits."""
    A, B, Xt = workloads.conditioned_batch(seed=66, count=5, n=300, kappa=1e3, nrhs=2)
    Xb, rb = solve_mixed(A, B)
    for s in (0, 3):
        Xs, rs = solve_mixed(A[s:s + 1], B[s:s + 1])
        assert np.array_equal(Xs[0], Xb[s]), s
        assert rs["iters"][0] == rb["iters"][s]


def test_pivoted_flag_keeps_the_step_kernels(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=67, count=3, n=200, kappa=1e4, nrhs=2)
    Xp, rp = solve_mixed(A, B, X_true=Xt, pivoted=True)
    _check(oracle, A, B, Xt, Xp, rp, 1e4)


# GMRES refinement (Carson and Higham's GMRES-IR on the same FP32 factors)

@pytest.mark.parametrize("n", [256, 640])
@pytest.mark.parametrize("kappa", [1e6, 1e8])
def test_gmres_high_kappa(lib, oracle, n, kappa):
    """kappa 1e6 (where plain refinement stalls): no fallback. kappa 1e8
    (kappa * u_fp32 > 1): every system at the bar, the FP64 fallback allowed
    for the systems whose first corrections do not contract."""
    A, B, Xt = workloads.conditioned_batch(seed=90 + n + int(np.log10(kappa)), count=4, n=n, kappa=kappa, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, gmres=True, max_iter=10)
    _check(oracle, A, B, Xt, X, rep, kappa, fallback_ok=kappa > 1e6)


def test_gmres_easy_and_multi_rhs(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=93, count=3, n=300, kappa=1e2, nrhs=1)
    X, rep = solve_mixed(A, B, X_true=Xt, gmres=True)
    _check(oracle, A, B, Xt, X, rep, 1e2)
    A, B, Xt = workloads.conditioned_batch(seed=94, count=3, n=384, kappa=1e6, nrhs=5)
    X, rep = solve_mixed(A, B, X_true=Xt, gmres=True)
    _check(oracle, A, B, Xt, X, rep, 1e6)


def test_gmres_row_scaled(lib, oracle):
    A, B, Xt = workloads.conditioned_batch(seed=95, count=4, n=256, kappa=1e4, nrhs=4, row_scale_decades=6)
    X, rep = solve_mixed(A, B, X_true=Xt, gmres=True)
    _check(oracle, A, B, Xt, X, rep, 1e4)


def test_gmres_alone_and_in_a_batch_agree_bitwise(lib):
    A, B, Xt = workloads.conditioned_batch(seed=96, count=4, n=300, kappa=1e6, nrhs=2)
    Xb, rb = solve_mixed(A, B, gmres=True)
    for s in (0, 2):
        Xs, rs = solve_mixed(A[s:s + 1], B[s:s + 1], gmres=True)
        assert np.array_equal(Xs[0], Xb[s]), s
        assert rs["iters"][0] == rb["iters"][s]


def test_gmres_rejects_pivoted(lib):
    A, B, _ = workloads.conditioned_batch(seed=97, count=1, n=64, kappa=1e2, nrhs=1)
    with pytest.raises(Exception):
        solve_mixed(A, B, gmres=True, pivoted=True)
