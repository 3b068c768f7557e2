"""Serving loop: continuous batching of factor and re-solve requests with
resident factors, against the C oracle of the reference."""
import threading

import numpy as np
import pytest

from numpp_b200 import _lib
from numpp_b200.serving import Server

from test_gpu_parity import check_solution

pytestmark = pytest.mark.gpu


def _system(rng, n, k, shift=True):
    A = rng.standard_normal((n, n)) + (n * np.eye(n) if shift else 0.0)
    return A, rng.standard_normal((n, k))


def test_factor_and_resolve_requests(lib, oracle):
    rng = np.random.default_rng(50)
    sizes = [(8, 1), (20, 3), (33, 1), (64, 8), (100, 2), (257, 1), (600, 5), (1030, 1), (31, 64), (129, 40)]
    with Server(budget_bytes=2 << 30, window_us=2000.0) as srv:
        reqs = []
        for i, (n, k) in enumerate(sizes):
            A, B = _system(rng, n, k)
            rid, X, fid = srv.submit(A, B, keep=(i % 2 == 0))
            reqs.append((rid, A, B, X, fid))
        # re-solves on the kept factors, possibly in the same batch as their factorisation
        resolves = []
        for rid, A, B, X, fid in reqs:
            if fid is not None:
                B2 = rng.standard_normal((A.shape[0], 3))
                r2, X2, _ = srv.submit(None, B2, factor=fid)
                resolves.append((r2, A, B2, X2))
        for rid, A, B, X, fid in reqs:
            rc, info, lat = srv.wait(rid)
            assert rc == 0 and info == 0 and lat > 0
            Xo, ok = oracle.solve(A[None], B[None])
            check_solution(X[None], Xo, A[None])
        for r2, A, B2, X2 in resolves:
            rc, info, lat = srv.wait(r2)
            assert rc == 0
            Xo, _ = oracle.solve(A[None], B2[None])
            check_solution(X2[None], Xo, A[None])
        st = srv.stats()
        assert st["completed"] == len(reqs) + len(resolves)
        assert st["resident"] == 5


def test_same_result_alone_and_in_a_mixed_batch(lib):
    """A request's arithmetic depends on its own order and right-hand sides only."""
    rng = np.random.default_rng(51)
    A, B = _system(rng, 300, 3, shift=False)
    with Server(budget_bytes=1 << 30, window_us=100.0) as srv:
        rid, X_alone, _ = srv.submit(A, B)
        assert srv.wait(rid)[0] == 0
    # orders 129..512 share a lane: the request runs in one batch with 200 and 300
    others = [_system(rng, n, k, shift=False) for n, k in [(40, 2), (700, 1), (12, 4), (300, 64), (200, 9), (90, 1)]]
    with Server(budget_bytes=1 << 30, window_us=50000.0) as srv:
        ids = [srv.submit(Ao, Bo)[0] for Ao, Bo in others[:3]]
        rid, X_mix, _ = srv.submit(A, B)
        ids += [srv.submit(Ao, Bo)[0] for Ao, Bo in others[3:]]
        assert srv.wait(rid)[0] == 0
        for i in ids:
            assert srv.wait(i)[0] == 0
        assert srv.stats()["batches"] == 3  # one per lane
    assert np.array_equal(X_alone, X_mix)


def test_least_recently_used_factor_is_evicted(lib, oracle):
    rng = np.random.default_rng(52)
    n = 1200  # 11.5 MB per factor: the arena of a 48 MB budget holds three
    with Server(budget_bytes=48 << 20, window_us=50.0) as srv:
        fids, systems = [], []
        for _ in range(4):
            A, B = _system(rng, n, 1)
            rid, X, fid = srv.submit(A, B, keep=True)
            assert srv.wait(rid)[0] == 0
            fids.append(fid)
            systems.append(A)
        assert srv.stats()["evictions"] >= 1
        B2 = rng.standard_normal((n, 2))
        rid, X2, _ = srv.submit(None, B2, factor=fids[0])  # the oldest: evicted
        assert srv.wait(rid)[0] == _lib.E_RANGE
        rid, X3, _ = srv.submit(None, B2, factor=fids[-1])
        assert srv.wait(rid)[0] == 0
        check_solution(X3[None], oracle.solve(systems[-1][None], B2[None])[0], systems[-1][None])
        srv.release(fids[-1])
        assert srv.stats()["resident"] <= 2


def test_singular_request_reports_info_and_keeps_nothing(lib):
    with Server(budget_bytes=256 << 20, window_us=50.0) as srv:
        A = np.zeros((50, 50))
        rid, X, fid = srv.submit(A, np.ones((50, 1)), keep=True)
        rc, info, _ = srv.wait(rid)
        assert rc == 0 and info == 1
        assert srv.stats()["resident"] == 0
        with pytest.raises(Exception):
            srv.submit(None, np.ones((50, 1)), factor=fid)


def test_concurrent_clients(lib, oracle):
    rng = np.random.default_rng(53)
    work = [_system(rng, int(n), int(k)) for n, k in zip(rng.integers(16, 400, 48), rng.integers(1, 9, 48))]
    results = [None] * len(work)
    with Server(budget_bytes=1 << 30, window_us=300.0, max_batch=16) as srv:
        def client(lo):
            for i in range(lo, len(work), 4):
                A, B = work[i]
                rid, X, _ = srv.submit(A, B)
                rc, info, _ = srv.wait(rid)
                results[i] = (rc, X)
        threads = [threading.Thread(target=client, args=(t,)) for t in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        assert srv.stats()["completed"] == len(work)
    for (A, B), (rc, X) in zip(work, results):
        assert rc == 0
        check_solution(X[None], oracle.solve(A[None], B[None])[0], A[None])
