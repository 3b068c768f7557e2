"""The benchmark workloads at their full sizes, checked through the C ABI.

The oracle (the C restatement of the reference's unblocked LU) finishes only
the smaller orders in seconds, so at full size the checks are the
size-independent ones, with oracle parity on a sample:

* uneven FP64 batch (8192 systems, n log-uniform [4, 512], nrhs {1, 8, 32},
  A = N(0,1) + n I, solve + slogdet for all, inverse for 10%): every system's
  normwise backward error computed on the device, and a 256-system sample
  against the oracle at the parity bar (1e-12 * cond(A), signs bit-exact);
* mixed precision, FP32/TF32 factors + FP64 refinement: 8 x 4096 at
  kappa 1e2 and 1e4 (and with GMRES refinement at 1e4 and 1e6), 64 x 1024 at
  kappa 1e8 (plain and GMRES refinement) (A = Q1 diag(sigma) Q2^T, sigma
  log-spaced 1..kappa, b = A x_true): reported and independently recomputed
  backward error <= 1e-10, forward error <= 10 * kappa * 1e-10, solutions
  against the FP64 LU (pivots bit-exact with the oracle up to 4096) and, for
  one 1024 system, against the oracle;
* BF16 factors after equilibration, 512 x 256, nrhs 4, rows scaled by
  10^U(-6, 6), kappa 1e1 and 1e3: every system ends at <= 1e-10 (refined, or
  refactored in FP64 where refinement stalled, and flagged as such).

The orthogonal factors of the conditioned matrices come from torch's seeded
generator and QR on the GPU (a NumPy QR of 16 matrices of order 4096 takes
minutes); the matrices themselves are float64 like every other input.
"""
import numpy as np
import pytest

from numpp_b200 import _lib, workloads
from numpp_b200.grouped import solve_grouped

from test_gpu_parity import check_solution

pytestmark = pytest.mark.gpu
P = _lib.ptr
TOL = 1e-10


def _torch():
    return pytest.importorskip("torch")


def _conditioned(torch, count, n, kappa, nrhs, seed, row_decades=0.0):
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    q1 = torch.linalg.qr(torch.randn(count, n, n, dtype=torch.float64, device=dev, generator=g))[0]
    q2 = torch.linalg.qr(torch.randn(count, n, n, dtype=torch.float64, device=dev, generator=g))[0]
    sig = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device=dev)
    A = (q1 * sig) @ q2.transpose(1, 2)
    del q1, q2
    if row_decades:
        A *= 10.0 ** (torch.rand(count, n, 1, dtype=torch.float64, device=dev, generator=g) * 2 * row_decades
                      - row_decades)
    A = A.contiguous()
    Xt = torch.randn(count, n, nrhs, dtype=torch.float64, device=dev, generator=g)
    return A, (A @ Xt).contiguous(), Xt


def _backward_error(A, B, X):
    """per system ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf), max-norm over columns."""
    R = B - A @ X
    return (R.abs().amax((1, 2)) / (A.abs().sum(2).amax(1) * X.abs().amax((1, 2)) + B.abs().amax((1, 2))))


def _mixed(lib, torch, A, B, Xt, flags=0, tol=TOL, max_iter=30):
    count, n, nrhs = B.shape
    dev = A.device
    X = torch.zeros_like(B)
    info = torch.zeros(count, dtype=torch.int32, device=dev)
    berr = torch.zeros(count, dtype=torch.float64, device=dev)
    ferr = torch.zeros_like(berr)
    iters = torch.zeros(count, dtype=torch.int32, device=dev)
    fb = torch.zeros_like(iters)
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_solve_mixed_batched(count, n, nrhs, P(A), P(B), P(X), P(Xt), tol, max_iter, flags, P(info),
                                        P(berr), P(ferr), P(iters), P(fb), st)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return X, {"info": info.cpu().numpy(), "berr": berr.cpu().numpy(), "ferr": ferr.cpu().numpy(),
               "iters": iters.cpu().numpy(), "fallback": fb.cpu().numpy()}


def _fp64(lib, torch, A, B):
    count, n, nrhs = B.shape
    X = torch.zeros_like(B)
    info = torch.zeros(count, dtype=torch.int32, device=A.device)
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_linalg_batched(count, n, nrhs, _lib.WANT_SOLVE, P(A), P(B), P(X), None, None, None, None,
                                   None, None, P(info), st)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert not info.any().item()
    return X


@pytest.mark.parametrize("kappa,gmres", [(1e2, False), (1e4, False), (1e4, True), (1e6, True)])
def test_mixed_8x4096(lib, kappa, gmres):
    """Plain refinement at kappa 1e2 must not fall back; at 1e4 a system whose
    block-pivoted factors grew too much may stall and is then refactored in
    FP64 (flagged); with GMRES refinement no system may fall back at 1e4 or 1e6."""
    torch = _torch()
    A, B, Xt = _conditioned(torch, 8, 4096, kappa, 1, seed=4096 + int(np.log10(kappa)))
    X, rep = _mixed(lib, torch, A, B, Xt, flags=_lib.MIXED_GMRES if gmres else 0)
    assert not rep["info"].any()
    assert np.all(rep["berr"] <= TOL), rep["berr"]
    if gmres or kappa <= 1e2:
        assert np.all(rep["fallback"] == 0), rep
    eta = _backward_error(A, B, X).cpu().numpy()
    assert np.all(eta <= TOL), eta  # the reported figure, recomputed independently
    # (a residual of 1e-12 relative is mostly cancellation: the two sums agree to a few digits)
    np.testing.assert_allclose(eta, rep["berr"], rtol=1e-2, atol=1e-16)
    assert np.all(rep["ferr"] <= 10 * kappa * TOL), rep["ferr"]
    X64 = _fp64(lib, torch, A, B)
    rel = ((X - X64).abs().amax((1, 2)) / X64.abs().amax((1, 2))).cpu().numpy()
    assert np.all(rel <= 10 * kappa * TOL), rel


@pytest.mark.parametrize("gmres", [False, True])
def test_mixed_64x1024_kappa1e8(lib, oracle, gmres):
    """kappa * u_fp32 > 1: plain refinement cannot be relied on; every system
    must still end at the bar, by refinement or by the flagged FP64
    refactorisation; with GMRES refinement too (the fallback count is reported)."""
    torch = _torch()
    kappa = 1e8
    A, B, Xt = _conditioned(torch, 64, 1024, kappa, 1, seed=1024 + 8)
    X, rep = _mixed(lib, torch, A, B, Xt, flags=_lib.MIXED_GMRES if gmres else 0)
    assert not rep["info"].any()
    assert np.all(rep["berr"] <= TOL), rep["berr"]
    eta = _backward_error(A, B, X).cpu().numpy()
    assert np.all(eta <= TOL), eta
    assert np.all(rep["ferr"] <= 10 * kappa * TOL), rep["ferr"]
    # one system against the oracle (the reference's LU restated)
    A0, B0 = A[:1].cpu().numpy(), B[:1].cpu().numpy()
    Xo, ok = oracle.solve(A0, B0)
    assert ok.all()
    rel = np.abs(X[:1].cpu().numpy() - Xo).max() / np.abs(Xo).max()
    assert rel <= 10 * kappa * TOL, rel


@pytest.mark.parametrize("kappa", [1e1, 1e3])
def test_bf16_row_scaled_512x256(lib, oracle, kappa):
    torch = _torch()
    A, B, Xt = _conditioned(torch, 512, 256, kappa, 4, seed=256 + int(kappa), row_decades=6.0)
    X, rep = _mixed(lib, torch, A, B, Xt, flags=_lib.MIXED_BF16)
    assert not rep["info"].any()
    assert np.all(rep["berr"] <= TOL), rep["berr"]
    eta = _backward_error(A, B, X).cpu().numpy()
    assert np.all(eta <= TOL), eta
    if kappa <= 1e1:  # kappa * u_bf16 << 1 after equilibration: refinement converges everywhere
        assert np.all(rep["fallback"] == 0), int(rep["fallback"].sum())
    refined = rep["fallback"] == 0
    assert np.all(rep["iters"][refined] >= 1)
    idx = np.arange(0, 512, 64)
    Xo, ok = oracle.solve(A[idx].cpu().numpy(), B[idx].cpu().numpy())
    assert ok.all()
    rel = np.abs(X[idx].cpu().numpy() - Xo).max(axis=(1, 2)) / np.abs(Xo).max(axis=(1, 2))
    assert np.all(rel <= 10 * kappa * TOL), rel


def test_uneven_8192_full_batch(lib, oracle):
    torch = _torch()
    sys_ = workloads.uneven_batch(seed=2025, count=8192)
    flags = _lib.WANT_SOLVE | _lib.WANT_SLOGDET | _lib.WANT_INV
    X, Inv, _, Sign, Logabs, info = solve_grouped(sys_, flags)
    assert not info.any()
    # every system: backward error on the device, grouped by order
    dev = torch.device("cuda:0")
    worst = 0.0
    for n in np.unique(sys_["n"]):
        for k in np.unique(sys_["nrhs"][sys_["n"] == n]):
            idx = np.nonzero((sys_["n"] == n) & (sys_["nrhs"] == k))[0]
            a = np.stack([sys_["A"][sys_["a_off"][i]:sys_["a_off"][i] + n * n] for i in idx]).reshape(-1, n, n)
            b = np.stack([sys_["B"][sys_["b_off"][i]:sys_["b_off"][i] + n * k] for i in idx]).reshape(-1, n, k)
            x = np.stack([X[sys_["b_off"][i]:sys_["b_off"][i] + n * k] for i in idx]).reshape(-1, n, k)
            eta = _backward_error(torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev),
                                  torch.from_numpy(x).to(dev))
            worst = max(worst, float(eta.max().item()))
    assert worst <= 1e-13, worst
    # parity with the oracle on a seeded sample
    idx = np.sort(np.random.default_rng(7).choice(8192, 256, replace=False))
    sub = workloads.take(sys_, idx)
    Xo, so, lo, invo, ok = oracle.solve_grouped(sub)
    assert ok.all()
    for j, i in enumerate(idx):
        n, k = int(sys_["n"][i]), int(sys_["nrhs"][i])
        A = sys_["A"][sys_["a_off"][i]:sys_["a_off"][i] + n * n].reshape(1, n, n)
        x = X[sys_["b_off"][i]:sys_["b_off"][i] + n * k].reshape(1, n, k)
        xo = Xo[sub["b_off"][j]:sub["b_off"][j] + n * k].reshape(1, n, k)
        check_solution(x, xo, A)
        assert Sign[i] == so[j], i
        cond = np.linalg.cond(A[0])
        assert abs(Logabs[i] - lo[j]) <= 1e-12 * cond * max(1.0, abs(lo[j])), i
        if sys_["inv_off"][i] >= 0:
            inv = Inv[sys_["inv_off"][i]:sys_["inv_off"][i] + n * n].reshape(1, n, n)
            invr = invo[sub["inv_off"][j]:sub["inv_off"][j] + n * n].reshape(1, n, n)
            check_solution(inv, invr, A)
