"""The linalg mirror on device-resident stacks, handed over through DLPack.

``solve``, ``inv``, ``det``, ``slogdet``, ``cholesky`` and ``matmul_batched`` take any tensor
that speaks the DLPack protocol (``__dlpack__`` / ``__dlpack_device__``) and
lives on the current CUDA device -- a torch tensor, a CuPy array, ... -- and
return torch tensors on the same device. The stacks never visit the host: the
DLTensor descriptors go straight to ``nppb_dl_linalg`` / ``nppb_dl_cholesky`` /
``nppb_dl_matmul``
(include/numpp_b200_dlpack.h), which enqueue on torch's current stream.

Semantics follow numpp_b200.linalg (NumPP's front-end, linalg.cpp:366-439 and
batched.cpp:75-108): b is a stack of vectors when b.ndim == a.ndim - 1, the
computation is float64 and float32 inputs come back float32, a singular matrix
raises ``LinAlgError("Singular matrix")`` in solve / inv. That check reads the
per-system info back (one small device-to-host copy and a wait); pass
``check=False`` to get ``(result, info)`` with nothing synchronised.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .linalg import Declined, LinAlgError, _check

_GetPointer = C.pythonapi.PyCapsule_GetPointer
_GetPointer.restype = C.c_void_p
_GetPointer.argtypes = [C.py_object, C.c_char_p]
_IsValid = C.pythonapi.PyCapsule_IsValid
_IsValid.restype = C.c_int
_IsValid.argtypes = [C.py_object, C.c_char_p]

_KDLCUDA = 2


def _torch():
    import torch
    return torch


class _Handoff:
    """DLPack capsules of one call's tensors, kept alive until the call returns."""

    def __init__(self, stream: int):
        self.stream = stream
        self.caps = []

    def ptr(self, t):
        if t is None:
            return None
        torch = _torch()
        if isinstance(t, torch.Tensor):
            cap = torch.utils.dlpack.to_dlpack(t)
        else:
            cap = t.__dlpack__(stream=self.stream)
        if not _IsValid(cap, b"dltensor"):
            raise TypeError("expected a legacy DLPack capsule named 'dltensor'")
        self.caps.append(cap)
        return _GetPointer(cap, b"dltensor")  # DLManagedTensor starts with its DLTensor


def _as_torch(x):
    """A torch view of a DLPack-capable CUDA tensor (zero-copy; torch.from_dlpack
    asks the producer to order its work before torch's current stream)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        t = x
    else:
        if not hasattr(x, "__dlpack_device__"):
            raise TypeError("expected a DLPack tensor on a CUDA device; host arrays go through numpp_b200.linalg")
        if x.__dlpack_device__()[0] != _KDLCUDA:
            raise Declined("not a CUDA tensor: host arrays go through numpp_b200.linalg")
        t = torch.from_dlpack(x)
    if t.device.type != "cuda":
        raise Declined("not a CUDA tensor: host arrays go through numpp_b200.linalg")
    if t.is_complex():
        raise Declined("complex dtypes are served by NumPP's portable CPU path, not the B200 path")
    return t


def _f64(t):
    torch = _torch()
    return t.to(torch.float64).contiguous()


def _out_dtype(*ts):
    torch = _torch()
    return torch.float32 if all(t.dtype == torch.float32 for t in ts) else torch.float64


def _call_linalg(flags, a, b=None, want_info=True):
    torch = _torch()
    stream = torch.cuda.current_stream(a.device).cuda_stream
    A = _f64(a)
    if A.dim() < 2 or A.shape[-1] != A.shape[-2]:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    lead = tuple(A.shape[:-2])
    out = {}
    B = _f64(b) if b is not None else None
    if flags & _lib.WANT_SOLVE:
        out["x"] = torch.empty_like(B)
    if flags & _lib.WANT_INV:
        out["inv"] = torch.empty_like(A)
    if flags & _lib.WANT_DET:
        out["det"] = torch.empty(lead, dtype=torch.float64, device=A.device)
    if flags & _lib.WANT_SLOGDET:
        out["sign"] = torch.empty(lead, dtype=torch.float64, device=A.device)
        out["logabs"] = torch.empty(lead, dtype=torch.float64, device=A.device)
    info = torch.zeros(lead, dtype=torch.int32, device=A.device) if want_info else None
    h = _Handoff(stream)
    L = _lib.load()
    with torch.cuda.device(A.device):
        _check(L.nppb_dl_linalg(flags, h.ptr(A), h.ptr(B), h.ptr(out.get("x")), h.ptr(out.get("inv")),
                                h.ptr(out.get("det")), h.ptr(out.get("sign")), h.ptr(out.get("logabs")),
                                h.ptr(info), stream))
    return out, info


def _vector_rule(a, b):
    if b.dim() == a.dim() - 1:
        if tuple(b.shape) != tuple(a.shape[:-1]):
            raise ValueError(f"solve: b has shape {tuple(b.shape)}, expected {tuple(a.shape[:-1])}")
    elif b.dim() == a.dim():
        if tuple(b.shape[:-1]) != tuple(a.shape[:-1]):
            raise ValueError(f"solve: b has shape {tuple(b.shape)}, expected {tuple(a.shape[:-1])} + (k,)")
    else:
        raise ValueError("solve: b.ndim must be a.ndim - 1 or a.ndim")


def solve(a, b, check=True):
    """x = a^-1 b on the device (linalg.cpp:368-385; stacks batched.cpp:90-100)."""
    a, b = _as_torch(a), _as_torch(b)
    if a.dim() < 2 or a.shape[-1] != a.shape[-2]:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    _vector_rule(a, b)
    out, info = _call_linalg(_lib.WANT_SOLVE, a, b)
    x = out["x"].to(_out_dtype(a, b))
    if not check:
        return x, info
    if bool(info.any()):
        raise LinAlgError("Singular matrix")
    return x


def inv(a, check=True):
    """a^-1 on the device (linalg.cpp:386-392; stacks batched.cpp:75)."""
    a = _as_torch(a)
    out, info = _call_linalg(_lib.WANT_INV, a)
    r = out["inv"].to(_out_dtype(a))
    if not check:
        return r, info
    if bool(info.any()):
        raise LinAlgError("Singular matrix")
    return r


def det(a):
    """det on the device (linalg.cpp:393-407): 0 for a singular matrix."""
    a = _as_torch(a)
    out, _ = _call_linalg(_lib.WANT_DET, a, want_info=False)
    return out["det"].to(_out_dtype(a))


def slogdet(a):
    """(sign, log|det|) on the device (linalg.cpp:408-439): (0, -inf) for a singular matrix."""
    a = _as_torch(a)
    out, _ = _call_linalg(_lib.WANT_SLOGDET, a, want_info=False)
    dt = _out_dtype(a)
    return out["sign"].to(dt), out["logabs"].to(dt)


def matmul_batched(a, b):
    """Stacked product lead + (m, k) @ lead + (k, n) on the device (the same lead
    on both; backend.cpp:121-177 for one matrix)."""
    torch = _torch()
    a, b = _as_torch(a), _as_torch(b)
    if a.dim() < 2 or b.dim() != a.dim():
        raise ValueError("matmul_batched: a and b need the same ndim >= 2")
    if a.shape[-1] != b.shape[-2] or a.shape[:-2] != b.shape[:-2]:
        raise ValueError("matmul: shape mismatch")
    stream = torch.cuda.current_stream(a.device).cuda_stream
    A, B = _f64(a), _f64(b)
    Cm = torch.empty(tuple(A.shape[:-1]) + (B.shape[-1],), dtype=torch.float64, device=A.device)
    h = _Handoff(stream)
    with torch.cuda.device(A.device):
        _check(_lib.load().nppb_dl_matmul(h.ptr(A), h.ptr(B), h.ptr(Cm), stream))
    return Cm.to(_out_dtype(a, b))


def cholesky(a, check=True):
    """Lower-triangular L with a = L L^T on the device (linalg.cpp:117-136; stacks
    batched.cpp:77), from a's lower triangle. ``LinAlgError("Matrix is not
    positive definite")`` if any matrix of the stack is not; ``check=False``
    returns ``(L, info)`` with nothing synchronised."""
    torch = _torch()
    a = _as_torch(a)
    if a.dim() < 2 or a.shape[-1] != a.shape[-2]:
        raise LinAlgError("Last 2 dimensions of the array must be square")
    stream = torch.cuda.current_stream(a.device).cuda_stream
    A = _f64(a)
    Lm = torch.empty_like(A)
    info = torch.zeros(tuple(A.shape[:-2]), dtype=torch.int32, device=A.device)
    h = _Handoff(stream)
    with torch.cuda.device(A.device):
        _check(_lib.load().nppb_dl_cholesky(h.ptr(A), h.ptr(Lm), h.ptr(info), stream))
    Lm = Lm.to(_out_dtype(a))
    if not check:
        return Lm, info
    if bool(info.any()):
        raise LinAlgError("Matrix is not positive definite")
    return Lm
