"""ctypes loaders for the two CPU checkers (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libnumpp_ref.so")
# NumPP's portable sources with the B200 front end and GPU vtable compiled in
# (the drop-in; oracle/Makefile target `dropin`)
DROPIN_SO = os.path.join(_HERE, "_ref", "dropin", "libnumpp_dropin.so")
# the reference's own CUDA backend (its GpuVTable gemm), for the a10 head-to-head
REFCUDA_SO = os.path.join(_HERE, "_ref", "refcuda", "libnumpp_refcuda.so")


def load_refcuda():
    """The reference's CUDA backend behind its C shim, or None when not built."""
    if not os.path.exists(REFCUDA_SO):
        return None
    L = C.CDLL(REFCUDA_SO)
    L.ref_cuda_available.restype = C.c_int
    L.ref_cuda_gemm.restype = C.c_int
    L.ref_cuda_gemm.argtypes = [C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
    return L

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)

F64 = 11  # numpp::DTypeId::Float64
F32 = 10  # numpp::DTypeId::Float32


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


def build_oracle(ref_src: str | None = None) -> None:
    """Compile liboracle.so, and the reference library when the NumPP source
    tree is named (``ref_src``, else the NUMPP_REF_SRC environment variable)
    and present; without one the reference build is skipped."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    src = ref_src or os.environ.get("NUMPP_REF_SRC")
    if src and os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "dropin", "refcuda", f"REF={src}"], check=True)


class Oracle:
    """The C restatement of the reference's portable LU path."""

    def __init__(self, path: str = _ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = C.CDLL(path)
        L.oracle_lu_decompose.argtypes = [_dp, C.c_int, _ip, _dp]
        L.oracle_solve.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int]
        L.oracle_inv.argtypes = [_dp, _dp, C.c_int]
        L.oracle_det.argtypes = [_dp, C.c_int]
        L.oracle_det.restype = C.c_double
        L.oracle_slogdet.argtypes = [_dp, C.c_int, _dp, _dp]
        L.oracle_matmul.argtypes = [C.c_int64, C.c_int64, C.c_int64, _dp, _dp, _dp]
        L.oracle_lu_batched.argtypes = [C.c_int64, C.c_int, _dp, _ip, _dp, _ip]
        L.oracle_solve_batched.argtypes = [C.c_int64, C.c_int, C.c_int, _dp, _dp, _dp, _ip]
        L.oracle_inv_batched.argtypes = [C.c_int64, C.c_int, _dp, _dp, _ip]
        L.oracle_det_batched.argtypes = [C.c_int64, C.c_int, _dp, _dp]
        L.oracle_slogdet_batched.argtypes = [C.c_int64, C.c_int, _dp, _dp, _dp]
        L.oracle_cholesky_batched.argtypes = [C.c_int64, C.c_int, _dp, _dp, _ip]
        L.oracle_lstsq.argtypes = [_dp, C.c_int, C.c_int, _dp, C.c_int, C.c_double, _dp, _dp, _ip, _dp]
        L.oracle_lstsq.restype = C.c_int
        L.oracle_solve_grouped.argtypes = [C.c_int64, _ip, _ip, _i64p, _i64p, _i64p,
                                           _dp, _dp, _dp, _dp, _dp, _dp, _ip]
        self.L = L

    # -- stacked (count, n, n) helpers; every array is float64 C-contiguous --
    def lu(self, A):
        A = np.array(A, dtype=np.float64, order="C", copy=True)
        cnt, n = A.shape[0], A.shape[-1]
        piv = np.zeros((cnt, n), np.intc)
        sgn = np.zeros(cnt)
        ok = np.zeros(cnt, np.intc)
        self.L.oracle_lu_batched(cnt, n, _ptr(A), _ptr(piv, _ip), _ptr(sgn), _ptr(ok, _ip))
        return A, piv, sgn, ok

    def solve(self, A, B):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        m = B.shape[-1] if B.ndim == 3 else 1
        X = np.zeros_like(B)
        ok = np.zeros(cnt, np.intc)
        self.L.oracle_solve_batched(cnt, n, m, _ptr(A), _ptr(B), _ptr(X), _ptr(ok, _ip))
        return X, ok

    def inv(self, A):
        A = np.ascontiguousarray(A, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        out = np.zeros_like(A)
        ok = np.zeros(cnt, np.intc)
        self.L.oracle_inv_batched(cnt, n, _ptr(A), _ptr(out), _ptr(ok, _ip))
        return out, ok

    def det(self, A):
        A = np.ascontiguousarray(A, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        out = np.zeros(cnt)
        self.L.oracle_det_batched(cnt, n, _ptr(A), _ptr(out))
        return out

    def slogdet(self, A):
        A = np.ascontiguousarray(A, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        s = np.zeros(cnt)
        la = np.zeros(cnt)
        self.L.oracle_slogdet_batched(cnt, n, _ptr(A), _ptr(s), _ptr(la))
        return s, la

    def lstsq(self, A, B, rcond=-1.0):
        """One 2-D problem: (x, residuals (size 0 or k), rank, singular values); B (m,) or (m, k)."""
        A = np.ascontiguousarray(A, np.float64)
        B = np.asarray(B, np.float64)
        bvec = B.ndim == 1
        Bm = np.ascontiguousarray(B.reshape(len(B), -1))
        m, n = A.shape
        k = Bm.shape[1]
        X = np.zeros((n, k))
        sv = np.zeros(min(m, n))
        rk = C.c_int()
        res = np.zeros(max(k, 1))
        has = self.L.oracle_lstsq(_ptr(A), m, n, _ptr(Bm), k, rcond, _ptr(X), _ptr(sv), C.byref(rk), _ptr(res))
        return (X[:, 0] if bvec else X), (res[:k] if has else np.zeros(0)), rk.value, sv

    def cholesky(self, A):
        """(count, n, n) stack -> (L, ok); ok[i] = 0 where matrix i is not positive definite."""
        A = np.ascontiguousarray(A, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        Lm = np.zeros_like(A)
        ok = np.zeros(cnt, np.intc)
        self.L.oracle_cholesky_batched(cnt, n, _ptr(A), _ptr(Lm), _ptr(ok, _ip))
        return Lm, ok

    def matmul(self, A, B):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        m, k = A.shape
        n = B.shape[1]
        Cm = np.zeros((m, n))
        self.L.oracle_matmul(m, n, k, _ptr(A), _ptr(B), _ptr(Cm))
        return Cm

    def matrix_power(self, A, p):
        """(count, n, n) stack to the integer power p, restating src/linalg/linalg.cpp:440-454
        per matrix (batched.cpp:83-84): the identity for p = 0, the inverse first for p < 0,
        then binary exponentiation with the p-order matmul. ok[i] = 0 when p < 0 and
        matrix i is singular (the reference raises linalg_error there)."""
        A = np.ascontiguousarray(A, np.float64)
        cnt, n = A.shape[0], A.shape[-1]
        R = np.zeros_like(A)
        ok = np.ones(cnt, np.intc)
        for i in range(cnt):
            if p < 0:
                base, o = self.inv(A[i:i + 1])
                base = base[0]
                ok[i] = o[0]
            else:
                base = A[i].copy()
            e = -p if p < 0 else p
            res = np.eye(n)
            while e > 0:
                if e & 1:
                    res = self.matmul(res, base)
                e >>= 1
                if e:
                    base = self.matmul(base, base)
            R[i] = res
        return R, ok

    def solve_grouped(self, sys, want_slogdet=True, want_inv=True):
        """sys: a packed uneven batch (numpp_b200 grouped layout as a dict of arrays)."""
        cnt = len(sys["n"])
        n = np.ascontiguousarray(sys["n"], np.intc)
        k = np.ascontiguousarray(sys["nrhs"], np.intc)
        X = np.zeros_like(sys["B"])
        s = np.zeros(cnt) if want_slogdet else None
        la = np.zeros(cnt) if want_slogdet else None
        inv = np.zeros(max(int(sys["inv_size"]), 1)) if want_inv else None
        ok = np.zeros(cnt, np.intc)
        self.L.oracle_solve_grouped(cnt, _ptr(n, _ip), _ptr(k, _ip), _ptr(sys["a_off"], _i64p),
                                    _ptr(sys["b_off"], _i64p), _ptr(sys["inv_off"], _i64p),
                                    _ptr(sys["A"]), _ptr(sys["B"]), _ptr(X), _ptr(s), _ptr(la),
                                    _ptr(inv), _ptr(ok, _ip))
        return X, s, la, inv, ok


class RefError(Exception):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class RefLib:
    """The reference's own public API (numpp::linalg / numpp::matmul)."""

    def __init__(self, path: str = _REF_SO):
        L = C.CDLL(path)
        vp = C.c_void_p
        cp = C.c_char_p
        L.ref_solve.argtypes = [C.c_int, _i64p, C.c_int, vp, C.c_int, _i64p, C.c_int, vp, vp,
                                _ip, _i64p, cp, C.c_int]
        L.ref_inv.argtypes = [C.c_int, _i64p, C.c_int, vp, vp, _ip, _i64p, cp, C.c_int]
        L.ref_det.argtypes = [C.c_int, _i64p, C.c_int, vp, vp, _ip, _i64p, cp, C.c_int]
        L.ref_slogdet.argtypes = [C.c_int, _i64p, C.c_int, vp, vp, vp, _ip, _i64p, cp, C.c_int]
        L.ref_matmul_cpu.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_int, vp, vp, vp, cp, C.c_int]
        L.ref_cholesky.argtypes = [C.c_int, _i64p, C.c_int, vp, vp, _ip, _i64p, cp, C.c_int]
        L.ref_lstsq.argtypes = [C.c_int, _i64p, vp, C.c_int, _i64p, vp, C.c_double, vp, _i64p, vp, _i64p, _i64p,
                                vp, _i64p, cp, C.c_int]
        L.ref_matrix_power.argtypes = [C.c_int, _i64p, C.c_int, vp, C.c_int64, vp, _ip, _i64p, cp,
                                       C.c_int]
        L.ref_tensorsolve.argtypes = [C.c_int, _i64p, C.c_int, vp, C.c_int, _i64p, C.c_int, vp, C.c_int,
                                      _i64p, vp, _ip, _i64p, cp, C.c_int]
        L.ref_tensorinv.argtypes = [C.c_int, _i64p, C.c_int, vp, C.c_int64, vp, _ip, _i64p, cp, C.c_int]
        L.ref_solve_grouped.argtypes = [C.c_int64, _i32p, _i32p, _i64p, _i64p, _i64p, _dp, _dp,
                                        _dp, _dp, _dp, _dp, _i32p, C.c_int]
        L.ref_standard_normal2.argtypes = [C.c_uint64, C.c_int64, _dp, C.c_int64, _dp]
        L.ref_uniform.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_int64, _dp]
        L.ref_last_backend.restype = C.c_int
        self.L = L

    BACKEND_CPU, BACKEND_CUDA = 1, 6

    def last_backend(self) -> int:
        """numpp::last_backend() of the calling thread, as its enum value."""
        return self.L.ref_last_backend()

    def clear_last_backend(self):
        self.L.ref_clear_last_backend()

    @staticmethod
    def _dt(a):
        if a.dtype == np.float64:
            return F64
        if a.dtype == np.float32:
            return F32
        raise TypeError(a.dtype)

    @staticmethod
    def _np(dt):
        return np.float64 if dt == F64 else np.float32

    def _call(self, fn, *args):
        err = C.create_string_buffer(256)
        rc = fn(*args, err, 256)
        if rc:
            raise RefError(rc, err.value.decode())

    def solve(self, A, B):
        A = np.ascontiguousarray(A)
        B = np.ascontiguousarray(B)
        sa = np.array(A.shape, np.int64)
        sb = np.array(B.shape, np.int64)
        out = np.zeros(B.size, np.float64)  # large enough for either dtype
        dt = C.c_int()
        sz = C.c_int64()
        self._call(self.L.ref_solve, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data, B.ndim,
                   _ptr(sb, _i64p), self._dt(B), B.ctypes.data, out.ctypes.data, C.byref(dt),
                   C.byref(sz))
        return np.frombuffer(out.tobytes(), self._np(dt.value), sz.value).reshape(B.shape)

    def _unary(self, fn, A, out_shape):
        A = np.ascontiguousarray(A)
        sa = np.array(A.shape, np.int64)
        out = np.zeros(max(int(np.prod(out_shape)), 1), np.float64)
        dt = C.c_int()
        sz = C.c_int64()
        self._call(fn, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data, out.ctypes.data,
                   C.byref(dt), C.byref(sz))
        return np.frombuffer(out.tobytes(), self._np(dt.value), sz.value).reshape(out_shape)

    def inv(self, A):
        return self._unary(self.L.ref_inv, A, A.shape)

    def det(self, A):
        return self._unary(self.L.ref_det, A, A.shape[:-2])

    def slogdet(self, A):
        A = np.ascontiguousarray(A)
        sa = np.array(A.shape, np.int64)
        shp = A.shape[:-2]
        cnt = max(int(np.prod(shp)), 1)
        s = np.zeros(cnt)
        la = np.zeros(cnt)
        dt = C.c_int()
        sz = C.c_int64()
        self._call(self.L.ref_slogdet, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data,
                   s.ctypes.data, la.ctypes.data, C.byref(dt), C.byref(sz))
        if dt.value == F32:
            s = np.frombuffer(s.tobytes(), np.float32, sz.value)
            la = np.frombuffer(la.tobytes(), np.float32, sz.value)
        return s[: sz.value].reshape(shp), la[: sz.value].reshape(shp)

    def matmul(self, A, B):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        Cm = np.zeros((A.shape[0], B.shape[1]))
        self._call(self.L.ref_matmul_cpu, A.shape[0], B.shape[1], A.shape[1], F64, A.ctypes.data,
                   B.ctypes.data, Cm.ctypes.data)
        return Cm

    def cholesky(self, A):
        return self._unary(self.L.ref_cholesky, A, A.shape)

    def lstsq(self, A, B, rcond=-1.0):
        A = np.ascontiguousarray(A, np.float64)
        B = np.ascontiguousarray(B, np.float64)
        sa = np.array(A.shape, np.int64)
        sb = np.array(B.shape, np.int64)
        X = np.zeros(max(A.shape[1] * (B.shape[1] if B.ndim == 2 else 1), 1))
        R = np.zeros(max(B.shape[1] if B.ndim == 2 else 1, 1))
        S = np.zeros(max(min(A.shape), 1))
        xs, rs, ss, rk = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        self._call(self.L.ref_lstsq, 2, _ptr(sa, _i64p), A.ctypes.data, B.ndim, _ptr(sb, _i64p), B.ctypes.data, rcond,
                   X.ctypes.data, C.byref(xs), R.ctypes.data, C.byref(rs), C.byref(rk), S.ctypes.data, C.byref(ss))
        xshape = (A.shape[1],) if B.ndim == 1 else (A.shape[1], B.shape[1])
        return X[:xs.value].reshape(xshape), R[:rs.value], rk.value, S[:ss.value]

    def matrix_power(self, A, p):
        A = np.ascontiguousarray(A)
        sa = np.array(A.shape, np.int64)
        out = np.zeros(max(A.size, 1), np.float64)
        dt = C.c_int()
        sz = C.c_int64()
        self._call(self.L.ref_matrix_power, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data, p,
                   out.ctypes.data, C.byref(dt), C.byref(sz))
        return np.frombuffer(out.tobytes(), self._np(dt.value), sz.value).reshape(A.shape)

    def tensorsolve(self, A, B, axes=()):
        """out shape: the unknown's shape, a.shape[b.ndim:] after the axes move."""
        A = np.ascontiguousarray(A)
        B = np.ascontiguousarray(B)
        sa = np.array(A.shape, np.int64)
        sb = np.array(B.shape, np.int64)
        ax = np.array(list(axes) or [0], np.int64)
        out = np.zeros(max(A.size, 1), np.float64)
        dt = C.c_int()
        sz = C.c_int64()
        self._call(self.L.ref_tensorsolve, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data, B.ndim,
                   _ptr(sb, _i64p), self._dt(B), B.ctypes.data, len(axes), _ptr(ax, _i64p),
                   out.ctypes.data, C.byref(dt), C.byref(sz))
        return np.frombuffer(out.tobytes(), self._np(dt.value), sz.value)

    def tensorinv(self, A, ind=2):
        """Flat result; its shape is a.shape[ind:] + a.shape[:ind]."""
        A = np.ascontiguousarray(A)
        sa = np.array(A.shape, np.int64)
        out = np.zeros(max(A.size, 1), np.float64)
        dt = C.c_int()
        sz = C.c_int64()
        self._call(self.L.ref_tensorinv, A.ndim, _ptr(sa, _i64p), self._dt(A), A.ctypes.data, ind,
                   out.ctypes.data, C.byref(dt), C.byref(sz))
        return np.frombuffer(out.tobytes(), self._np(dt.value), sz.value)

    def standard_normal2(self, seed, n1, n2):
        a = np.zeros(n1)
        b = np.zeros(n2)
        rc = self.L.ref_standard_normal2(seed, n1, _ptr(a), n2, _ptr(b))
        if rc:
            raise RefError(rc, "standard_normal failed")
        return a, b

    def uniform(self, seed, low, high, n):
        out = np.zeros(n)
        rc = self.L.ref_uniform(seed, low, high, n, _ptr(out))
        if rc:
            raise RefError(rc, "uniform failed")
        return out

    def solve_grouped(self, sys, want_slogdet=True, want_inv=True, threads=1):
        cnt = len(sys["n"])
        n = np.ascontiguousarray(sys["n"], np.int32)
        k = np.ascontiguousarray(sys["nrhs"], np.int32)
        X = np.zeros_like(sys["B"])
        s = np.zeros(cnt) if want_slogdet else None
        la = np.zeros(cnt) if want_slogdet else None
        inv = np.zeros(max(int(sys["inv_size"]), 1)) if want_inv else None
        ok = np.zeros(cnt, np.int32)
        self.L.ref_solve_grouped(cnt, _ptr(n, _i32p), _ptr(k, _i32p), _ptr(sys["a_off"], _i64p),
                                 _ptr(sys["b_off"], _i64p), _ptr(sys["inv_off"], _i64p),
                                 _ptr(sys["A"]), _ptr(sys["B"]), _ptr(X), _ptr(s), _ptr(la),
                                 _ptr(inv), _ptr(ok, _i32p), threads)
        return X, s, la, inv, ok


def load_oracle() -> Oracle:
    return Oracle()


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def load_ref() -> RefLib:
    return RefLib()
