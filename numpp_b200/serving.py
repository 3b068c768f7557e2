"""Client of the serving loop (continuous batching, resident factors) on the C ABI.

The server owns a worker thread on the device; `submit` returns at once and
`wait` blocks for one request. Buffers handed to `submit` are used in place
by the worker, so they stay referenced here until the request is waited for.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .linalg import _check


class ServerError(RuntimeError):
    pass


class Server:
    def __init__(self, budget_bytes: int = 8 << 30, window_us: float = 500.0, max_batch: int = 256):
        self._L = _lib.load()
        self._h = C.c_void_p()
        _check(self._L.nppb_server_create(C.byref(self._h), int(budget_bytes), float(window_us), int(max_batch)))
        self._keep = {}

    def submit(self, A, B, X=None, keep: bool = False, factor: int | None = None):
        """Factor A and solve (A given), or re-solve on a resident factor
        (A None, factor = its id). Returns (request id, X, factor id or None)."""
        B = np.ascontiguousarray(B, np.float64)
        if B.ndim == 1:
            B = B[:, None]
        n, k = B.shape
        X = np.empty_like(B) if X is None else X
        if A is not None:
            A = np.ascontiguousarray(A, np.float64)
            if A.shape != (n, n):
                raise ValueError(f"A is {A.shape}, B is {B.shape}")
        rid, fid = C.c_int64(-1), C.c_int64(-1)
        _check(self._L.nppb_server_submit(self._h, n, k, _lib.ptr(A), _lib.ptr(B), _lib.ptr(X),
                                          -1 if factor is None else int(factor), int(bool(keep)),
                                          C.byref(rid), C.byref(fid)))
        self._keep[rid.value] = (A, B, X)
        return rid.value, X, (fid.value if fid.value >= 0 else None)

    def wait(self, rid: int, timeout_s: float = 60.0):
        """(status, info, latency seconds) of a finished request."""
        info, lat = C.c_int32(0), C.c_double(0.0)
        rc = self._L.nppb_server_wait(self._h, int(rid), float(timeout_s), C.byref(info), C.byref(lat))
        if rc == _lib.DECLINED:
            raise ServerError(f"request {rid} did not finish within {timeout_s} s")
        self._keep.pop(rid, None)
        return rc, info.value, lat.value

    def release(self, factor: int) -> None:
        _check(self._L.nppb_server_release_factor(self._h, int(factor)))

    def stats(self) -> dict:
        out = (C.c_int64 * 6)()
        _check(self._L.nppb_server_stats(self._h, out))
        keys = ("completed", "batches", "resident", "resident_bytes", "evictions", "queued")
        return dict(zip(keys, list(out)))

    def close(self) -> None:
        if self._h:
            self._L.nppb_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
