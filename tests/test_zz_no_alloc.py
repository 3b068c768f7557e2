"""The allocation-free solve (nppb_d_solve_batched_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory while they run (hosts
whose device memory is reserved up front, fixed-pool allocators where a
cudaMalloc would fail or stall): its scratch is a fixed 32 MiB array inside the
library, shared by every call. Checked here:

* against the allocating solve (nppb_d_linalg_batched, NPPB_WANT_SOLVE) and
  against the oracle (the C restatement of the reference's LU), within the
  parity tolerance of the other tests, 1e-12 * cond(A);
* on two calls in a row, so that a call does not depend on what the previous
  one left in the shared array;
* on orders that take each route: the warp kernel (n <= 32, no scratch), the
  single-CTA panels (33..512) and the cluster panels with look-ahead (> 512);
* that a call takes nothing from the device's default memory pool (the pool
  the library's allocating entry points draw from): its in-use high-water
  mark, reset before the call, stays at or below the in-use figure from
  before it.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from numpp_b200 import _lib

pytestmark = pytest.mark.gpu
P = _lib.ptr

# CUmemPool_attribute values (CUDA driver API)
_USED_MEM_CURRENT = 7
_USED_MEM_HIGH = 8


class _DefaultPool:
    """The current device's default memory pool through the driver API."""

    def __init__(self, ordinal: int):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), ordinal) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr: int) -> int:
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = ctypes.c_uint64(0)  # the high-water mark can only be reset to zero
        assert self.cu.cuMemPoolSetAttribute(self.pool, _USED_MEM_HIGH, ctypes.byref(zero)) == 0


def _noalloc(lib, torch, dA, dB, count, n, k):
    dX = torch.full_like(dB, np.nan)
    info = torch.full((count,), -1, dtype=torch.int32, device=dB.device)
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nppb_d_solve_batched_noalloc(count, n, k, P(dA), P(dB), P(dX), P(info), st)
    assert rc == 0, _lib.last_error()
    return dX, info


@pytest.mark.parametrize("count,n,nrhs", [(64, 20, 3), (24, 100, 8), (6, 300, 2), (4, 512, 1), (2, 700, 2)])
def test_noalloc_matches_allocating_solve_and_oracle(lib, oracle, count, n, nrhs):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    pool = _DefaultPool(0)
    for call in range(2):  # two calls in a row on the shared scratch
        rng = np.random.default_rng(1000 * n + call)
        A = rng.standard_normal((count, n, n))
        B = rng.standard_normal((count, n, nrhs))
        dA = torch.from_numpy(A).to(dev)
        dB = torch.from_numpy(B).to(dev)
        torch.cuda.synchronize()
        used = pool.get(_USED_MEM_CURRENT)
        pool.reset_high()
        dX1, i1 = _noalloc(lib, torch, dA, dB, count, n, nrhs)
        torch.cuda.synchronize()
        # any allocation would lift the mark above the bytes already in use
        assert pool.get(_USED_MEM_HIGH) <= used, "the allocation-free solve drew from the memory pool"

        dX2 = torch.zeros_like(dB)
        i2 = torch.full((count,), -1, dtype=torch.int32, device=dev)
        st = torch.cuda.current_stream().cuda_stream
        rc = lib.nppb_d_linalg_batched(count, n, nrhs, _lib.WANT_SOLVE, P(dA), P(dB), P(dX2), None, None, None,
                                       None, None, None, P(i2), st)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        X1, X2 = dX1.cpu().numpy(), dX2.cpu().numpy()
        assert not i1.cpu().numpy().any() and not i2.cpu().numpy().any()
        Xo, ok = oracle.solve(A, B)
        assert ok.all()
        cond = np.linalg.cond(A)
        flat = lambda Z: Z.reshape(count, -1)  # noqa: E731
        for ref in (X2, Xo):
            err = np.linalg.norm(flat(X1 - ref), axis=1) / np.linalg.norm(flat(ref), axis=1)
            assert np.all(err <= 1e-12 * cond), (err / cond).max()


def test_noalloc_singular_system_reports_info(lib):
    """A zero pivot in one system sets its info and leaves the others solved,
    also when the previous call on the shared scratch had no failure."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    rng = np.random.default_rng(77)
    A = rng.standard_normal((3, 64, 64))
    A[1, :, 5] = 0.0  # column 5 of system 1: exact zero pivot at step 5
    B = rng.standard_normal((3, 64, 1))
    dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    dX, info = _noalloc(lib, torch, dA, dB, 3, 64, 1)
    torch.cuda.synchronize()
    i = info.cpu().numpy()
    assert i[0] == 0 and i[1] > 0 and i[2] == 0, i
    X = dX.cpu().numpy()
    for s in (0, 2):
        assert np.abs(A[s] @ X[s] - B[s]).max() < 1e-10


def test_noalloc_rejects_batches_beyond_its_scratch(lib):
    # 16 systems of order 512 need 16 * (8*512*512 + 8616) bytes > 32 MiB
    rc = lib.nppb_d_solve_batched_noalloc(16, 512, 1, 1, 1, 1, 1, None)
    assert rc == _lib.E_RANGE
    assert "32" in _lib.last_error() or "bytes" in _lib.last_error()
