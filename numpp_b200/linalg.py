"""numpp::linalg front-end on the B200 path (host-side mirror of NumPP's interface).

Same names, argument meaning and error behaviour as NumPP's
include/numpp/linalg/linalg.hpp:29-32 and src/backend/backend.cpp:121-177,
on numpy arrays:

* ``solve(a, b)``  -- linalg.cpp:368-385; stacked a (ndim > 2) follows
  batched.cpp:90-100: b is a stack of vectors when b.ndim == a.ndim - 1
  (NumPP keeps NumPy 1.x's rule), else a stack of (n, k) matrices.
* ``inv(a)``, ``det(a)``, ``slogdet(a)`` -- linalg.cpp:386-439, batched.cpp:75-108.
* ``matmul(a, b)`` -- backend.cpp:121-177 with the GPU forced (2-D only).
* ``matmul_batched(a, b)`` -- equal-batch (..., m, k) @ (..., k, n) on the
  batched DMMA GEMM. The reference has no stacked matmul (backend.cpp:122
  rejects ndim != 2); this is the product its stacked ``matrix_power`` runs per
  matrix, offered as one call. Leading axes broadcast as in numpy.matmul.
* ``cholesky(a)`` -- linalg.cpp:117-136, stacks batched.cpp:77: the lower
  triangle of a is read, ``LinAlgError("Matrix is not positive definite")``.
* ``matrix_power(a, n)`` -- linalg.cpp:440-454, stacks batched.cpp:83-84.
* ``tensorsolve(a, b, axes)``, ``tensorinv(a, ind)`` -- tensor_solve.cpp:10-49.
* ``cond(a, p)`` -- tensor.cpp:359-393: p in {1, -1, inf, -inf, "fro"} as
  norm(a, p) * norm(inv(a), p), inf when a is singular; p None / 2 / -2 from
  the singular values.
* ``lstsq(a, b, rcond)`` -- linalg.cpp:755-784 (its Jacobi SVD :620-712):
  solution, residuals, rank, singular values; ``svdvals(a)`` -- :725.

dtype policy (``la_kind``, linalg.cpp:20-26): the computation is float64;
float32 results come back as float32, every other real dtype as float64.
Complex inputs are not served by this path (NumPP's portable CPU kernel keeps
them), so they raise ``Declined``.

Errors: ``LinAlgError("Last 2 dimensions of the array must be square")`` and
``LinAlgError("Singular matrix")`` as numpp::linalg_error (linalg.cpp:30-33,
100, 110); a singular matrix makes det 0 and slogdet (0, -inf) (:402, :418-423).
Like the reference loop, one singular matrix in a stack fails the whole solve /
inv call. Unlike the reference, an empty stack returns an empty result (the
reference indexes its first output there) and mismatched right-hand-side shapes
raise ``ValueError`` before any device work.

All GPU work goes through the C ABI (``_lib``); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class LinAlgError(Exception):
    """numpp::linalg_error (include/numpp/core/error.hpp:43-46)."""


class Declined(NotImplementedError):
    """The request is outside the B200 path (the GpuVTable slot would return false)."""


class DeviceError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"numpp_b200 error {code}: {msg}")
        self.code = code


def _check(rc: int) -> None:
    if rc == _lib.OK:
        return
    if rc == _lib.DECLINED:
        raise Declined(_lib.last_error() or "declined")
    raise DeviceError(rc, _lib.last_error())


class NativeBackend:
    """The C ABI on host buffers: (count, n, n) float64 stacks in, numpy out."""

    def __init__(self):
        self.L = _lib.load()

    def solve(self, A, B):
        cnt, n = A.shape[0], A.shape[-1]
        k = B.shape[-1]
        X = np.empty_like(B)
        info = np.zeros(cnt, np.int32)
        _check(self.L.nppb_solve_batched(cnt, n, k, _lib.ptr(A), _lib.ptr(B), _lib.ptr(X),
                                         _lib.ptr(info)))
        return X, info

    def inv(self, A):
        cnt, n = A.shape[0], A.shape[-1]
        out = np.empty_like(A)
        info = np.zeros(cnt, np.int32)
        _check(self.L.nppb_inv_batched(cnt, n, _lib.ptr(A), _lib.ptr(out), _lib.ptr(info)))
        return out, info

    def det(self, A):
        cnt, n = A.shape[0], A.shape[-1]
        out = np.empty(cnt)
        _check(self.L.nppb_det_batched(cnt, n, _lib.ptr(A), _lib.ptr(out)))
        return out

    def slogdet(self, A):
        cnt, n = A.shape[0], A.shape[-1]
        s = np.empty(cnt)
        la = np.empty(cnt)
        _check(self.L.nppb_slogdet_batched(cnt, n, _lib.ptr(A), _lib.ptr(s), _lib.ptr(la)))
        return s, la

    def gemm(self, A, B):
        m, k = A.shape
        n = B.shape[1]
        Cm = np.empty((m, n), A.dtype)
        dt = _lib.DT_FLOAT64 if A.dtype == np.float64 else _lib.DT_FLOAT32
        _check(self.L.nppb_gemm(dt, m, n, k, _lib.ptr(A), _lib.ptr(B), _lib.ptr(Cm)))
        return Cm


    def cholesky(self, A):
        cnt, n = A.shape[0], A.shape[-1]
        Lm = np.empty_like(A)
        info = np.zeros(cnt, np.int32)
        _check(self.L.nppb_cholesky_batched(cnt, n, _lib.ptr(A), _lib.ptr(Lm), _lib.ptr(info)))
        return Lm, info

    def lstsq(self, A, B, rcond):
        """A (count, m, n), B (count, m, k) -> X, S, rank, resid, has_resid."""
        cnt, m, n = A.shape
        k = B.shape[-1]
        X = np.empty((cnt, n, k))
        S = np.empty((cnt, min(m, n)))
        rank = np.zeros(cnt, np.int32)
        res = np.zeros((cnt, max(k, 1)))
        has = np.zeros(cnt, np.int32)
        _check(self.L.nppb_lstsq_batched(cnt, m, n, k, _lib.ptr(A), _lib.ptr(B), float(rcond), _lib.ptr(X),
                                         _lib.ptr(S), _lib.ptr(rank), _lib.ptr(res), _lib.ptr(has)))
        return X, S, rank, res[:, :k], has

    def svdvals(self, A):
        cnt, m, n = A.shape
        S = np.empty((cnt, min(m, n)))
        rank = np.zeros(cnt, np.int32)
        _check(self.L.nppb_lstsq_batched(cnt, m, n, 0, _lib.ptr(A), None, -1.0, None, _lib.ptr(S), _lib.ptr(rank),
                                         None, None))
        return S

    def gemm_batched(self, A, B):
        cnt, m, k = A.shape
        n = B.shape[-1]
        Cm = np.empty((cnt, m, n))
        _check(self.L.nppb_gemm_batched(cnt, m, n, k, _lib.ptr(A), _lib.ptr(B), _lib.ptr(Cm)))
        return Cm

    def matrix_power(self, A, p):
        cnt, n = A.shape[0], A.shape[-1]
        R = np.empty_like(A)
        info = np.zeros(cnt, np.int32)
        _check(self.L.nppb_matrix_power_batched(cnt, n, p, _lib.ptr(A), _lib.ptr(R), _lib.ptr(info)))
        return R, info


_default = None


def default_backend():
    global _default
    if _default is None:
        _default = NativeBackend()
    return _default


def _la_out(dt) -> np.dtype:
    dt = np.dtype(dt)
    if dt.kind == "c":
        raise Declined("complex dtypes are served by NumPP's portable CPU path, not the B200 path")
    if dt.kind not in "biuf":
        raise TypeError(f"unsupported dtype {dt}")
    return np.dtype(np.float32) if dt == np.float32 else np.dtype(np.float64)


def _require_square(a) -> None:
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise LinAlgError("Last 2 dimensions of the array must be square")


def _stack(a):
    """(lead shape, count, n, (count, n, n) float64 contiguous) of a stack."""
    if a.shape[-1] != a.shape[-2]:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    lead = a.shape[:-2]
    n = a.shape[-1]
    cnt = int(np.prod(lead)) if lead else 1
    A3 = np.ascontiguousarray(a, dtype=np.float64).reshape(cnt, n, n)
    return lead, cnt, n, A3


def solve(a, b, backend=None):
    be = backend or default_backend()
    a = np.asarray(a)
    b = np.asarray(b)
    out_dt = _la_out(np.result_type(a.dtype, b.dtype))
    if a.ndim > 2:
        lead, cnt, n, A3 = _stack(a)
        bvec = b.ndim == a.ndim - 1
        k = 1 if bvec else b.shape[-1]
        if b.size != cnt * n * k or b.shape[-2 if not bvec else -1] != n:
            raise ValueError(f"solve: b of shape {b.shape} does not match a of shape {a.shape}")
        B3 = np.ascontiguousarray(b, dtype=np.float64).reshape(cnt, n, k)
        out_shape = lead + ((n,) if bvec else (n, k))
    else:
        _require_square(a)
        n = a.shape[0]
        bvec = b.ndim == 1
        if b.ndim not in (1, 2) or b.shape[0] != n:
            raise ValueError(f"solve: b of shape {b.shape} does not match a of shape {a.shape}")
        k = 1 if bvec else b.shape[1]
        A3 = np.ascontiguousarray(a, dtype=np.float64).reshape(1, n, n)
        B3 = np.ascontiguousarray(b, dtype=np.float64).reshape(1, n, k)
        cnt = 1
        out_shape = b.shape
    if cnt == 0 or n == 0 or k == 0:
        return np.zeros(out_shape, out_dt)
    X, info = be.solve(A3, B3)
    if np.any(info):
        raise LinAlgError("Singular matrix")
    return X.reshape(out_shape).astype(out_dt, copy=False)


def inv(a, backend=None):
    be = backend or default_backend()
    a = np.asarray(a)
    out_dt = _la_out(a.dtype)
    if a.ndim > 2:
        lead, cnt, n, A3 = _stack(a)
    else:
        _require_square(a)
        lead, cnt, n = (), 1, a.shape[0]
        A3 = np.ascontiguousarray(a, dtype=np.float64).reshape(1, n, n)
    if cnt == 0 or n == 0:
        return np.zeros(lead + (n, n), out_dt)
    out, info = be.inv(A3)
    if np.any(info):
        raise LinAlgError("Singular matrix")
    return out.reshape(lead + (n, n)).astype(out_dt, copy=False)


def det(a, backend=None):
    be = backend or default_backend()
    a = np.asarray(a)
    out_dt = _la_out(a.dtype)
    if a.ndim > 2:
        lead, cnt, n, A3 = _stack(a)
    else:
        _require_square(a)
        lead, cnt, n = (), 1, a.shape[0]
        A3 = np.ascontiguousarray(a, dtype=np.float64).reshape(1, n, n)
    if cnt == 0:
        return np.zeros(lead, out_dt)
    return be.det(A3).reshape(lead).astype(out_dt, copy=False)


def slogdet(a, backend=None):
    """(sign, logabsdet), numpp::linalg::SignLogDet (linalg.hpp:22)."""
    be = backend or default_backend()
    a = np.asarray(a)
    out_dt = _la_out(a.dtype)
    if a.ndim > 2:
        lead, cnt, n, A3 = _stack(a)
    else:
        _require_square(a)
        lead, cnt, n = (), 1, a.shape[0]
        A3 = np.ascontiguousarray(a, dtype=np.float64).reshape(1, n, n)
    if cnt == 0:
        return np.zeros(lead, out_dt), np.zeros(lead, out_dt)
    s, la = be.slogdet(A3)
    return (s.reshape(lead).astype(out_dt, copy=False),
            la.reshape(lead).astype(out_dt, copy=False))


def matmul(a, b, backend=None):
    """numpp::matmul(a, b, Backend::Cuda) for float32 / float64 2-D operands."""
    be = backend or default_backend()
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim != 2 or b.ndim != 2:
        raise ValueError("matmul requires 2-D arrays")
    if a.shape[1] != b.shape[0]:
        raise ValueError("matmul: shape mismatch")
    dt = np.result_type(a.dtype, b.dtype)
    if dt not in (np.float32, np.float64):
        raise Declined(f"the B200 gemm serves float32 and float64, not {dt}")
    if a.shape[0] == 0 or b.shape[1] == 0:
        return np.zeros((a.shape[0], b.shape[1]), dt)
    return be.gemm(np.ascontiguousarray(a, dt), np.ascontiguousarray(b, dt))


def matmul_batched(a, b, backend=None):
    """Stacked float64 product (..., m, k) @ (..., k, n); leading axes broadcast.

    2-D operands are numpp::matmul itself (backend.cpp:121-177). Float32 and
    every other real dtype compute in float64 and return float64 (float32 stays
    float32), like the linalg front-end's dtype policy."""
    be = backend or default_backend()
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim < 2 or b.ndim < 2:
        raise ValueError("matmul requires at least 2-D arrays")
    if a.shape[-1] != b.shape[-2]:
        raise ValueError("matmul: shape mismatch")
    out = _la_out(np.result_type(a.dtype, b.dtype))
    lead = np.broadcast_shapes(a.shape[:-2], b.shape[:-2])
    m, k, n = a.shape[-2], a.shape[-1], b.shape[-1]
    cnt = int(np.prod(lead)) if lead else 1
    if cnt == 0 or m == 0 or n == 0:
        return np.zeros(lead + (m, n), out)
    A3 = np.ascontiguousarray(np.broadcast_to(a, lead + (m, k)), np.float64).reshape(cnt, m, k)
    B3 = np.ascontiguousarray(np.broadcast_to(b, lead + (k, n)), np.float64).reshape(cnt, k, n)
    return be.gemm_batched(A3, B3).reshape(lead + (m, n)).astype(out, copy=False)


def matrix_power(a, n, backend=None):
    """numpp::linalg::matrix_power (linalg.cpp:440-454; stacks batched.cpp:83-84).

    n = 0 gives the identity, n < 0 inverts first (``LinAlgError("Singular
    matrix")`` when a matrix of the stack is singular), then binary
    exponentiation: the same sequence of products as the reference."""
    be = backend or default_backend()
    a = np.asarray(a)
    out = _la_out(a.dtype)
    if a.ndim < 2:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    n = int(n)
    if not -(1 << 63) <= n < (1 << 63):
        raise OverflowError("matrix_power exponent out of int64 range")
    lead, cnt, d, A3 = _stack(a)
    if cnt == 0 or d == 0:
        return np.zeros(a.shape, out)
    R, info = be.matrix_power(A3, n)
    if n < 0 and info.any():
        raise LinAlgError("Singular matrix")
    return R.reshape(a.shape).astype(out, copy=False)


def tensorsolve(a, b, axes=None, backend=None):
    """numpy/NumPP tensorsolve (tensor_solve.cpp:10-34): the named axes of a move
    to the end, the trailing a.ndim - b.ndim axes form the unknown's shape, and
    the square reshape of a is solved against b.ravel()."""
    a = np.asarray(a)
    b = np.asarray(b)
    an = a.ndim
    if axes:
        allaxes = list(range(an))
        for k in axes:
            if k not in allaxes:
                raise ValueError(f"tensorsolve: axis {k} is not an axis of a")
            allaxes.remove(k)
            allaxes.append(k)
        a = a.transpose(allaxes)
    bn = b.ndim
    if an < bn:
        raise LinAlgError("tensorsolve: a.ndim must be >= b.ndim")
    oldshape = a.shape[bn:]
    prod = int(np.prod(oldshape)) if oldshape else 1
    if a.size != prod * prod:
        raise LinAlgError("tensorsolve: prod(a.shape[b.ndim:]) must equal prod(a.shape[:b.ndim])")
    if b.size != prod:
        raise ValueError("tensorsolve: b does not reshape to the unknown's size")
    x = solve(a.reshape(prod, prod), b.reshape(prod), backend=backend)
    return x.reshape(oldshape)


def tensorinv(a, ind=2, backend=None):
    """numpy/NumPP tensorinv (tensor_solve.cpp:36-49): inv of a reshaped to
    (prod(a.shape[ind:]), prod(a.shape[:ind])), result shape a.shape[ind:] + a.shape[:ind]."""
    a = np.asarray(a)
    nd = a.ndim
    ind = int(ind)
    if ind <= 0 or ind > nd:
        raise ValueError("Invalid ind argument")
    sh = a.shape
    prod = int(np.prod(sh[ind:])) if sh[ind:] else 1
    lead = int(np.prod(sh[:ind]))
    return inv(a.reshape(prod, lead), backend=backend).reshape(sh[ind:] + sh[:ind])


def _matrix_norm(x, p):
    ax = np.abs(x)
    if p == "fro":
        return np.sqrt((x * x).sum(axis=(-2, -1)))
    if p in (1, -1):
        col = ax.sum(axis=-2)
        return col.max(axis=-1) if p == 1 else col.min(axis=-1)
    row = ax.sum(axis=-1)
    return row.max(axis=-1) if p == np.inf else row.min(axis=-1)


def cond(a, p=None, backend=None):
    """numpp::cond (src/tensor/tensor.cpp:359-393) for the inverse-based norms.

    p in {1, -1, inf, -inf, "fro"}: norm(a, p) * norm(inv(a), p) in float64,
    inf for a singular matrix (the reference catches linalg_error). p None /
    2: s_max / s_min (inf when s_min is 0), p -2: s_min / s_max (0 when s_max
    is 0), from the singular values of ``svdvals`` (tensor.cpp:372-390). A
    stack (..., n, n) gives one number per matrix."""
    if p is None or (not isinstance(p, str) and p in (2, -2)):
        s = svdvals(a, backend=backend)
        if s.shape[-1] == 0:
            return np.zeros(s.shape[:-1]) if s.ndim > 1 else np.float64(0.0)
        hi, lo = s[..., 0], s[..., -1]
        with np.errstate(divide="ignore", invalid="ignore"):
            if p == -2:
                c = np.where(hi > 0, lo / np.where(hi > 0, hi, 1.0), 0.0)
            else:
                c = np.where(lo > 0, hi / np.where(lo > 0, lo, 1.0), np.inf)
        return c if c.ndim else np.float64(c)
    if isinstance(p, str):
        if p != "fro":
            raise ValueError(f"cond: unsupported norm {p!r}")
    elif p not in (1, -1, np.inf, -np.inf):
        raise ValueError(f"cond: unsupported norm {p!r}")
    be = backend or default_backend()
    a = np.asarray(a)
    _la_out(a.dtype)
    if a.ndim < 2:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    lead, cnt, n, A3 = _stack(a)
    if n == 0:
        raise LinAlgError("cond is not defined on empty arrays")
    if cnt == 0:
        return np.zeros(lead)
    Ai, info = be.inv(A3)
    c = _matrix_norm(A3, p) * _matrix_norm(Ai, p)
    c = np.where(info != 0, np.inf, c)
    return c.reshape(lead) if lead else np.float64(c[0])


def cholesky(a, backend=None):
    """numpp::linalg::cholesky (linalg.cpp:117-136; stacks batched.cpp:77).

    Lower-triangular L with a = L L^T, computed from a's lower triangle (the
    upper one is never read). One matrix of a stack that is not positive
    definite fails the whole call, as the reference loop does."""
    be = backend or default_backend()
    a = np.asarray(a)
    out = _la_out(a.dtype)
    if a.ndim < 2:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    lead, cnt, n, A3 = _stack(a)
    if cnt == 0 or n == 0:
        return np.zeros(a.shape, out)
    Lm, info = be.cholesky(A3)
    if info.any():
        raise LinAlgError("Matrix is not positive definite")
    return Lm.reshape(a.shape).astype(out, copy=False)


def svdvals(a, backend=None):
    """Singular values, descending, of a (..., m, n) stack (linalg.cpp:725;
    the reference's one-sided Jacobi SVD, :620-712)."""
    be = backend or default_backend()
    a = np.asarray(a)
    _la_out(a.dtype)
    if a.ndim < 2:
        raise ValueError("svdvals requires at least a 2-D array")
    lead, (m, n) = a.shape[:-2], a.shape[-2:]
    cnt = int(np.prod(lead)) if lead else 1
    if cnt == 0 or m == 0 or n == 0:
        return np.zeros(lead + (min(m, n),))
    A3 = np.ascontiguousarray(a, np.float64).reshape(cnt, m, n)
    return be.svdvals(A3).reshape(lead + (min(m, n),))


def lstsq(a, b, rcond=-1.0, backend=None):
    """numpp::linalg::lstsq (linalg.cpp:755-784): (solution, residuals, rank,
    singular values) of a 2-D a (m, n) and b (m,) or (m, k). Singular values
    at or below tol = (rcond < 0 ? eps * max(m, n) : rcond) * s_max are
    dropped; residuals (sum of squares per column) only when m > n and the
    rank is n, else an empty array. Shapes past the device limits (min(m, n)
    or k above 64, or a problem too large for one SM's shared memory) are
    ``Declined``."""
    be = backend or default_backend()
    a = np.asarray(a)
    b = np.asarray(b)
    if a.ndim != 2:
        raise LinAlgError("lstsq: a must be 2-D")
    m, n = a.shape
    bvec = b.ndim == 1
    if b.ndim not in (1, 2) or b.shape[0] != m:
        raise LinAlgError("lstsq: b must have a.shape[0] rows")
    out = _la_out(np.result_type(a.dtype, b.dtype))
    Bm = b.reshape(m, 1) if bvec else b
    k = Bm.shape[1]
    if m == 0 or n == 0 or k == 0:
        x = np.zeros((n,) if bvec else (n, k), out)
        return x, np.zeros(0), 0, np.zeros(min(m, n))
    A3 = np.ascontiguousarray(a, np.float64).reshape(1, m, n)
    B3 = np.ascontiguousarray(Bm, np.float64).reshape(1, m, k)
    X, S, rank, res, has = be.lstsq(A3, B3, rcond)
    x = X[0, :, 0] if bvec else X[0]
    resid = res[0] if has[0] else np.zeros(0)
    return x.astype(out, copy=False), resid, int(rank[0]), S[0]


def _main(argv=None):
    """Time the small uniform batch on the device: 256 systems of order 32,
    A = N(0,1) + 32 I from PCG64 (seed 2025), one right-hand side, solve + det
    in one call of nppb_d_linalg_batched (CUDA events over back-to-back calls)."""
    import argparse

    import torch

    from . import workloads
    p = argparse.ArgumentParser(prog="python -m numpp_b200.linalg")
    p.add_argument("--small", action="store_true", help="the 256 x 32 x 32 solve + det batch")
    p.add_argument("--reps", type=int, default=200)
    a = p.parse_args(argv)
    if not a.small:
        p.error("nothing to time: pass --small")
    L = _lib.load()
    P = _lib.ptr
    dev = torch.device("cuda:0")
    A, B = workloads.uniform_batch(seed=2025)
    dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    dX = torch.zeros_like(dB)
    det = torch.zeros(256, dtype=torch.float64, device=dev)
    info = torch.zeros(256, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream().cuda_stream

    def run():
        _check(L.nppb_d_linalg_batched(256, 32, 1, _lib.WANT_SOLVE | _lib.WANT_DET, P(dA), P(dB), P(dX), None,
                                       P(det), None, None, None, None, P(info), st))

    for _ in range(10):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        run()
    e1.record()
    e1.synchronize()
    print("256 x 32 x 32 solve + det: %.2f us per call (%d back-to-back calls)" % (e0.elapsed_time(e1) / a.reps * 1e3,
                                                                                  a.reps), flush=True)


if __name__ == "__main__":
    _main()
