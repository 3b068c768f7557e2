"""The allocation-free solve (nppb_d_solve_batched_noalloc) against the
allocating one (nppb_d_linalg_batched with NPPB_WANT_SOLVE), through the C ABI.

It exists for callers that cannot allocate device memory while they run (code
inside a CUDA graph capture, hosts with all device memory reserved up front):
its scratch is a fixed 32 MiB array inside the library, shared by every call.
Two calls in a row check that a call does not depend on what the previous one
left in that array. Same tolerance as the other parity tests: 1e-12 * cond(A).
"""
import numpy as np
import pytest

from numpp_b200 import _lib

pytestmark = pytest.mark.gpu
P = _lib.ptr


def _solve_both(lib, torch, A, B):
    dev = torch.device("cuda:0")
    count, n, k = B.shape[0], A.shape[-1], B.shape[-1]
    dA = torch.from_numpy(A).to(dev)
    dB = torch.from_numpy(B).to(dev)
    dX1 = torch.full_like(dB, np.nan)
    dX2 = torch.zeros_like(dB)
    i1 = torch.full((count,), -1, dtype=torch.int32, device=dev)
    i2 = torch.full((count,), -1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_solve_batched_noalloc(count, n, k, P(dA), P(dB), P(dX1), P(i1), st)
    assert rc == 0, _lib.last_error()
    rc = lib.nppb_d_linalg_batched(count, n, k, _lib.WANT_SOLVE, P(dA), P(dB), P(dX2), None, None, None,
                                   None, None, None, P(i2), st)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    return dX1.cpu().numpy(), dX2.cpu().numpy(), i1.cpu().numpy(), i2.cpu().numpy()


@pytest.mark.parametrize("count,n,nrhs", [(64, 20, 3), (24, 100, 8), (6, 300, 2), (4, 512, 1)])
def test_noalloc_matches_allocating_solve(lib, count, n, nrhs):
    torch = pytest.importorskip("torch")
    for call in range(2):  # two calls in a row on the shared scratch
        rng = np.random.default_rng(1000 * n + call)
        A = rng.standard_normal((count, n, n))
        B = rng.standard_normal((count, n, nrhs))
        X1, X2, i1, i2 = _solve_both(lib, torch, A, B)
        assert not i1.any() and not i2.any()
        cond = np.linalg.cond(A)
        err = np.linalg.norm((X1 - X2).reshape(count, -1), axis=1) / np.linalg.norm(X2.reshape(count, -1), axis=1)
        assert np.all(err <= 1e-12 * cond), (err / cond).max()
        resid = np.abs(np.einsum("bij,bjk->bik", A, X1) - B).max()
        assert resid < 1e-8 * cond.max()


def test_noalloc_rejects_batches_beyond_its_scratch(lib):
    # 16 systems of order 512 need 16 * (8*512*512 + 8616) bytes > 32 MiB
    rc = lib.nppb_d_solve_batched_noalloc(16, 512, 1, 1, 1, 1, 1, None)
    assert rc == _lib.E_RANGE
    assert "32" in _lib.last_error() or "bytes" in _lib.last_error()
