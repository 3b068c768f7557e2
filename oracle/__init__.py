"""CPU oracle — TEST INFRASTRUCTURE ONLY.

Two checkers for the batched dense linear-solve path:

* ``lu_oracle.c`` (``liboracle.so``): a plain-C restatement of NumPP's portable
  LU / solve / inv / det / slogdet / matmul, each function citing the reference
  lines it follows.
* ``_ref/libnumpp_ref.so``: NumPP's own unmodified CPU sources compiled by
  ``oracle/Makefile`` plus ``ref_shim.cpp`` (extern "C" wrappers around the
  reference's public ``numpp::linalg`` / ``numpp::matmul`` calls). Present only
  where it was built (it is built here and shipped as a binary).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
legs may import this package, and only as the checker or the timed baseline.
The product (``numpp_b200``) never imports it.
"""
from .oracle import (  # noqa: F401
    Oracle,
    RefLib,
    load_oracle,
    load_ref,
    ref_available,
)
