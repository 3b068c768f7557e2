"""The two-level (blocked) factorisation of uniform batches: outer blocks of
128 columns, the trailing matrix updated once per block by a K = 128 DMMA GEMM
after the block's row moves and triangular solves. It is selected per process
by NPPB_BLOCKED_MIN_N, so each case runs in a child process with it set low
enough to cover partial blocks; results are held to the same bar as the
one-level path (x within 1e-12 * cond(A) of the oracle, pivots / signs exact)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from numpp_b200 import _lib
L = _lib.load()
cases = json.loads(sys.argv[2])
out = {}
for key, (cnt, n, k, inv, seed) in cases.items():
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((cnt, n, n)) + np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((cnt, n, k))
    X = np.empty_like(B)
    info = np.zeros(cnt, np.int32)
    assert L.nppb_solve_batched(cnt, n, k, _lib.ptr(A), _lib.ptr(B), _lib.ptr(X), _lib.ptr(info)) == 0, _lib.last_error()
    s = np.empty(cnt); la = np.empty(cnt)
    assert L.nppb_slogdet_batched(cnt, n, _lib.ptr(A), _lib.ptr(s), _lib.ptr(la)) == 0
    I = np.empty_like(A) if inv else None
    if inv:
        iinfo = np.zeros(cnt, np.int32)
        assert L.nppb_inv_batched(cnt, n, _lib.ptr(A), _lib.ptr(I), _lib.ptr(iinfo)) == 0
    np.save(sys.argv[3] + f"/{key}_X.npy", X)
    np.save(sys.argv[3] + f"/{key}_s.npy", s)
    np.save(sys.argv[3] + f"/{key}_la.npy", la)
    if inv:
        np.save(sys.argv[3] + f"/{key}_I.npy", I)
print("ok")
"""

CASES = {"a": (3, 200, 3, True, 1), "b": (2, 333, 1, True, 2), "c": (2, 1000, 8, False, 3),
         "d": (1, 1100, 2, True, 4), "e": (4, 129, 5, False, 5)}


def test_blocked_matches_oracle(lib, oracle, tmp_path):
    env = dict(os.environ, NPPB_BLOCKED_MIN_N="64")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(CASES), str(tmp_path)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]
    for key, (cnt, n, k, inv, seed) in CASES.items():
        rng = np.random.default_rng(seed)
        A = rng.standard_normal((cnt, n, n)) + np.sqrt(n) * np.eye(n)
        B = rng.standard_normal((cnt, n, k))
        X = np.load(tmp_path / f"{key}_X.npy")
        Xo, ok = oracle.solve(A, B)
        assert ok.all()
        cond = np.linalg.cond(A)
        err = np.linalg.norm((X - Xo).reshape(cnt, -1), axis=1)
        assert np.all(err <= 1e-12 * cond * np.linalg.norm(Xo.reshape(cnt, -1), axis=1)), (key, err)
        so, lo = oracle.slogdet(A)
        assert np.array_equal(np.load(tmp_path / f"{key}_s.npy"), so), key
        np.testing.assert_allclose(np.load(tmp_path / f"{key}_la.npy"), lo, rtol=1e-12)
        if inv:
            Io, _ = oracle.inv(A)
            I = np.load(tmp_path / f"{key}_I.npy")
            d = np.linalg.norm((I - Io).reshape(cnt, -1), axis=1)
            assert np.all(d <= 1e-12 * cond * np.linalg.norm(Io.reshape(cnt, -1), axis=1)), key
