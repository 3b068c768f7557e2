"""Mixed-precision batched solve (FP32 factors, FP64 refinement) on the C ABI."""
from __future__ import annotations

import numpy as np

from . import _lib
from .linalg import _check


_FACTOR = {"3xtf32": 0, "fp32": _lib.MIXED_FP32_FMA, "tf32": _lib.MIXED_TF32, "bf16": _lib.MIXED_BF16}


def solve_mixed(A, B, X_true=None, tol: float = 1e-10, max_iter: int = 10, equilibrate: bool = True,
                fallback: bool = True, factor: str = "3xtf32", tcgen05: bool = False, pivoted: bool = False,
                gmres: bool = False):
    """X for a (count, n, n) / (count, n, nrhs) float64 batch; returns
    (X, report) with report = dict(berr, ferr, iters, fallback, info) per system.

    Default: the blocked FP32 factorisation of the butterfly-transformed
    matrix (pivoting inside each 128-row diagonal block, triangular solves and
    trailing updates as tcgen05 GEMMs with error-compensated TF32 products).
    pivoted=True, or any factor other than "3xtf32", or tcgen05=True: LU with
    partial pivoting on the step-wise kernels, factor choosing the trailing
    products: "3xtf32" (error-compensated TF32, close to FP32), "tf32" or
    "bf16" (one tensor-core product), "fp32" (FMA); tcgen05: TF32 products on
    the tcgen05 tensor cores with TMEM accumulators instead of mma.sync.
    gmres=True (default factorisation only): each correction by GMRES
    preconditioned with the FP32 factorisation on FP64 vectors (GMRES-IR), for
    conditioning the plain refinement stalls on."""
    L = _lib.load()
    A = np.ascontiguousarray(A, np.float64)
    B = np.ascontiguousarray(B, np.float64)
    cnt, n, k = B.shape[0], A.shape[-1], B.shape[-1]
    X = np.zeros_like(B)
    info = np.zeros(cnt, np.int32)
    berr = np.zeros(cnt)
    ferr = np.full(cnt, np.nan)
    iters = np.zeros(cnt, np.int32)
    fb = np.zeros(cnt, np.int32)
    Xt = None if X_true is None else np.ascontiguousarray(X_true, np.float64)
    flags = ((0 if equilibrate else _lib.MIXED_NO_EQUILIBRATE) | (0 if fallback else _lib.MIXED_NO_FALLBACK)
             | _FACTOR[factor] | (_lib.MIXED_TCGEN05 if tcgen05 else 0) | (_lib.MIXED_PIVOTED if pivoted else 0)
             | (_lib.MIXED_GMRES if gmres else 0))
    P = _lib.ptr
    _check(L.nppb_solve_mixed_batched(cnt, n, k, P(A), P(B), P(X), P(Xt), tol, max_iter, flags, P(info),
                                      P(berr), P(ferr), P(iters), P(fb)))
    return X, {"berr": berr, "ferr": ferr, "iters": iters, "fallback": fb, "info": info}


def _main(argv=None):
    """Time the mixed solve on a device-resident conditioned batch:
    A = Q1 diag(sigma) Q2^T (Q from QR of N(0,1) matrices, sigma log-spaced
    1..kappa), b = A x_true, one right-hand side; prints the time, the
    corrections and the fallbacks of each repetition (CUDA events)."""
    import argparse

    import torch

    p = argparse.ArgumentParser(prog="python -m numpp_b200.mixed")
    p.add_argument("--count", type=int, default=64)
    p.add_argument("--n", type=int, default=1024)
    p.add_argument("--kappa", type=float, default=1e2)
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--gmres", action="store_true")
    p.add_argument("--pivoted", action="store_true")
    a = p.parse_args(argv)
    L = _lib.load()
    P = _lib.ptr
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev)
    g.manual_seed(a.n)
    q1 = torch.linalg.qr(torch.randn(a.count, a.n, a.n, dtype=torch.float64, device=dev, generator=g))[0]
    q2 = torch.linalg.qr(torch.randn(a.count, a.n, a.n, dtype=torch.float64, device=dev, generator=g))[0]
    sig = torch.logspace(0.0, float(np.log10(a.kappa)), a.n, dtype=torch.float64, device=dev)
    A = ((q1 * sig) @ q2.transpose(1, 2)).contiguous()
    del q1, q2
    xt = torch.randn(a.count, a.n, 1, dtype=torch.float64, device=dev, generator=g)
    B = (A @ xt).contiguous()
    X = torch.zeros_like(B)
    info = torch.zeros(a.count, dtype=torch.int32, device=dev)
    be = torch.zeros(a.count, dtype=torch.float64, device=dev)
    fe = torch.zeros_like(be)
    it = torch.zeros_like(info)
    fb = torch.zeros_like(info)
    flags = (_lib.MIXED_GMRES if a.gmres else 0) | (_lib.MIXED_PIVOTED if a.pivoted else 0)
    st = torch.cuda.current_stream().cuda_stream

    def run():
        _check(L.nppb_d_solve_mixed_batched(a.count, a.n, 1, P(A), P(B), P(X), P(xt), 1e-10, 30, flags, P(info),
                                            P(be), P(fe), P(it), P(fb), st))

    run()
    torch.cuda.synchronize()
    for _ in range(a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        e1.synchronize()
        print("%d x %d kappa %.0e: %.3f ms, corrections max %d, fallbacks %d, max backward error %.2e"
              % (a.count, a.n, a.kappa, e0.elapsed_time(e1), it.max().item(), fb.sum().item(), be.max().item()),
              flush=True)


if __name__ == "__main__":
    _main()
