"""B200-native (sm_100a) batched dense linear-solve path for NumPP.

``numpp_b200.linalg`` mirrors numpp::linalg::{solve, inv, det, slogdet} and
numpp::matmul on numpy arrays; ``numpp_b200.grouped.Plan`` runs uneven batches.
Everything executes through libnumpp_b200.so (C ABI: include/numpp_b200.h);
importing works without it, the first call raises if it is missing.
"""
from . import _lib  # noqa: F401
from .linalg import (  # noqa: F401
    Declined,
    DeviceError,
    LinAlgError,
    det,
    inv,
    matmul,
    slogdet,
    solve,
)

__all__ = ["solve", "inv", "det", "slogdet", "matmul", "LinAlgError", "Declined", "DeviceError"]
