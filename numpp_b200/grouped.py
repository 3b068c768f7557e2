"""Uneven batches through the plan entry points of the C ABI (nppb_plan_*)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .linalg import _check


class Plan:
    """Size-classed, graph-replayed execution of a packed uneven batch.

    ``sys`` is the packed layout of ``workloads.uneven_batch`` (n, nrhs, a_off,
    b_off, inv_off); ``flags`` a ``_lib.WANT_*`` mask.
    """

    def __init__(self, sys: dict, flags: int):
        self.L = _lib.load()
        self.count = int(len(sys["n"]))
        self._keep = [np.ascontiguousarray(sys["n"], np.int32), np.ascontiguousarray(sys["nrhs"], np.int32),
                      np.ascontiguousarray(sys["a_off"], np.int64), np.ascontiguousarray(sys["b_off"], np.int64),
                      np.ascontiguousarray(sys["inv_off"], np.int64)]
        h = C.c_void_p()
        _check(self.L.nppb_plan_create(C.byref(h), self.count, *(_lib.ptr(x) for x in self._keep), flags))
        self.h = h
        self.flags = flags
        a, b, i = C.c_int64(), C.c_int64(), C.c_int64()
        _check(self.L.nppb_plan_sizes(self.h, C.byref(a), C.byref(b), C.byref(i)))
        self.a_elems, self.b_elems, self.inv_elems = a.value, b.value, i.value

    def execute(self, A, B, X, Inv, Det, Sign, Logabs, info, stream=None):
        """Device buffers (torch tensors or raw addresses); enqueues on `stream`."""
        args = [_lib.ptr(x) for x in (A, B, X, Inv, Det, Sign, Logabs, info)]
        st = stream if isinstance(stream, int) or stream is None else stream.cuda_stream
        _check(self.L.nppb_plan_execute(self.h, *args, st))

    def autotune(self, A, B, X, Inv, Det, Sign, Logabs, info, stream=None):
        """Keep the fastest chain count and look-ahead setting for these device
        buffers; returns (chains, look-ahead on, ms per execution)."""
        st = stream if isinstance(stream, int) or stream is None else stream.cuda_stream
        ch, ms = C.c_int32(0), C.c_float(0.0)
        _check(self.L.nppb_plan_autotune(self.h, *(_lib.ptr(x) for x in (A, B, X, Inv, Det, Sign, Logabs, info)),
                                         st, C.byref(ch), C.byref(ms)))
        return abs(ch.value), ch.value < 0, ms.value

    def execute_host(self, A, B, X=None, Inv=None, Det=None, Sign=None, Logabs=None, info=None):
        """Host buffers (numpy); returns once the outputs are back."""
        _check(self.L.nppb_plan_execute_host(self.h, *(_lib.ptr(x) for x in (A, B, X, Inv, Det, Sign, Logabs, info))))

    def classes(self):
        """[(kernel, order bound, systems, flops, bytes)] per size class."""
        out = []
        for c in range(self.L.nppb_plan_num_classes(self.h)):
            w, b, s = C.c_int(), C.c_int(), C.c_int64()
            f, by = C.c_double(), C.c_double()
            _check(self.L.nppb_plan_class_info(self.h, c, C.byref(w), C.byref(b), C.byref(s), C.byref(f),
                                               C.byref(by)))
            out.append(("warp" if w.value else "cta", b.value, s.value, f.value, by.value))
        return out

    def time_classes(self, A, B, X, Inv, Det, Sign, Logabs, info, stream=None, reps=3):
        """Mean ms of one launch of each class, CUDA events on `stream`."""
        nc = self.L.nppb_plan_num_classes(self.h)
        ms = (C.c_float * max(nc, 1))()
        st = stream if isinstance(stream, int) or stream is None else stream.cuda_stream
        _check(self.L.nppb_plan_time_classes(self.h, *(_lib.ptr(x) for x in (A, B, X, Inv, Det, Sign, Logabs, info)),
                                             st, reps, ms))
        return [ms[i] for i in range(nc)]

    KINDS = ("warp_lu", "panel", "update", "back")

    def launches(self) -> int:
        """Kernel launches per execution (nodes of the replayed graph)."""
        return int(self.L.nppb_plan_num_launches(self.h))

    def time_kernels(self, A, B, X, Inv, Det, Sign, Logabs, info, stream=None):
        """{kind: (ms, flops)} summed over the launches of one execution."""
        ms = (C.c_double * 4)()
        fl = (C.c_double * 4)()
        st = stream if isinstance(stream, int) or stream is None else stream.cuda_stream
        _check(self.L.nppb_plan_time_kernels(self.h, *(_lib.ptr(x) for x in (A, B, X, Inv, Det, Sign, Logabs, info)),
                                             st, ms, fl))
        return {k: (ms[i], fl[i]) for i, k in enumerate(self.KINDS)}

    def close(self):
        if getattr(self, "h", None):
            self.L.nppb_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_grouped(sys: dict, flags: int = _lib.WANT_SOLVE | _lib.WANT_SLOGDET | _lib.WANT_INV):
    """One-shot host call: returns X, inverses, det, sign, logabsdet, info (numpy)."""
    L = _lib.load()
    cnt = len(sys["n"])
    X = np.zeros_like(sys["B"])
    Inv = np.zeros(max(int(sys["inv_size"]), 1))
    Det, Sign, Logabs = np.zeros(cnt), np.zeros(cnt), np.zeros(cnt)
    info = np.zeros(cnt, np.int32)
    keep = [np.ascontiguousarray(sys["n"], np.int32), np.ascontiguousarray(sys["nrhs"], np.int32),
            np.ascontiguousarray(sys["a_off"], np.int64), np.ascontiguousarray(sys["b_off"], np.int64),
            np.ascontiguousarray(sys["inv_off"], np.int64)]
    A = np.ascontiguousarray(sys["A"], np.float64)
    B = np.ascontiguousarray(sys["B"], np.float64)
    _check(L.nppb_solve_grouped(cnt, *(_lib.ptr(x) for x in keep), flags, _lib.ptr(A), _lib.ptr(B),
                                _lib.ptr(X), _lib.ptr(Inv), _lib.ptr(Det), _lib.ptr(Sign), _lib.ptr(Logabs),
                                _lib.ptr(info)))
    return X, Inv, Det, Sign, Logabs, info
