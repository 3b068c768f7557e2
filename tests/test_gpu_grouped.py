"""Uneven batches through the plan entry points vs the oracle; the full-size
8192-system batch through size-independent checks (backward error, slogdet)."""
import numpy as np
import pytest

from numpp_b200 import _lib, workloads
from numpp_b200.grouped import Plan, solve_grouped

pytestmark = pytest.mark.gpu
FLAGS = _lib.WANT_SOLVE | _lib.WANT_SLOGDET | _lib.WANT_INV | _lib.WANT_DET


def per_system(sys, X):
    for i in range(len(sys["n"])):
        n, k = int(sys["n"][i]), int(sys["nrhs"][i])
        A = sys["A"][sys["a_off"][i]:sys["a_off"][i] + n * n].reshape(n, n)
        B = sys["B"][sys["b_off"][i]:sys["b_off"][i] + n * k].reshape(n, k)
        x = X[sys["b_off"][i]:sys["b_off"][i] + n * k].reshape(n, k)
        yield i, A, B, x


def check_vs_oracle(sys, X, Inv, Det, Sign, Logabs, info, oracle):
    Xo, so, lo, invo, ok = oracle.solve_grouped(sys)
    assert np.array_equal(info == 0, ok == 1)
    assert np.array_equal(Sign, so)
    for i, A, B, x in per_system(sys, X):
        n, k = A.shape[0], B.shape[1]
        cond = np.linalg.cond(A) if n else 1.0
        xo = Xo[sys["b_off"][i]:sys["b_off"][i] + n * k]
        assert np.linalg.norm(x.ravel() - xo) <= 1e-12 * cond * max(np.linalg.norm(xo), 1e-300)
        assert abs(Logabs[i] - lo[i]) <= 1e-12 * cond * max(abs(lo[i]), 1.0)
        if sys["inv_off"][i] >= 0:
            o = sys["inv_off"][i]
            d = Inv[o:o + n * n] - invo[o:o + n * n]
            assert np.linalg.norm(d) <= 1e-12 * cond * max(np.linalg.norm(invo[o:o + n * n]), 1e-300)
    fin = Logabs < 700.0   # det overflows to +-inf past e^709; compare where it is finite
    np.testing.assert_allclose(Det[fin], Sign[fin] * np.exp(Logabs[fin]), rtol=1e-9)
    assert np.all(np.isinf(Det[~fin]) | (np.abs(Det[~fin]) > 1e300))


def test_one_shot_uneven(lib, oracle):
    sys = workloads.uneven_batch(seed=11, count=300, n_lo=1, n_hi=512, nrhs_choices=(1, 8, 32),
                                 inv_fraction=0.2)
    X, Inv, Det, Sign, Logabs, info = solve_grouped(sys, FLAGS)
    check_vs_oracle(sys, X, Inv, Det, Sign, Logabs, info, oracle)


def test_plan_host_replay(lib, oracle):
    sys = workloads.uneven_batch(seed=12, count=200, n_lo=1, n_hi=300, nrhs_choices=(1, 3, 8))
    plan = Plan(sys, FLAGS)
    cnt = len(sys["n"])
    outs = None
    for _ in range(3):  # graph captured once, replayed
        X = np.zeros_like(sys["B"])
        Inv = np.zeros(max(plan.inv_elems, 1))
        Det, Sign, Logabs = np.zeros(cnt), np.zeros(cnt), np.zeros(cnt)
        info = np.full(cnt, -1, np.int32)
        plan.execute_host(sys["A"], sys["B"], X, Inv, Det, Sign, Logabs, info)
        if outs is None:
            outs = (X, Inv, Det, Sign, Logabs, info)
            check_vs_oracle(sys, X, Inv, Det, Sign, Logabs, info, oracle)
        else:
            for a, b in zip(outs, (X, Inv, Det, Sign, Logabs, info)):
                assert np.array_equal(a, b)  # deterministic replay
    plan.close()


def test_plan_device_buffers_torch(lib, oracle):
    torch = pytest.importorskip("torch")
    sys = workloads.uneven_batch(seed=13, count=120, n_lo=2, n_hi=200)
    plan = Plan(sys, FLAGS)
    dev = torch.device("cuda:0")
    cnt = len(sys["n"])
    dA = torch.from_numpy(sys["A"]).to(dev)
    dB = torch.from_numpy(sys["B"]).to(dev)
    dX = torch.zeros_like(dB)
    dInv = torch.zeros(max(plan.inv_elems, 1), dtype=torch.float64, device=dev)
    d = [torch.zeros(cnt, dtype=torch.float64, device=dev) for _ in range(3)]
    dinfo = torch.zeros(cnt, dtype=torch.int32, device=dev)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        plan.execute(dA, dB, dX, dInv, d[0], d[1], d[2], dinfo, stream=s)
    s.synchronize()
    check_vs_oracle(sys, dX.cpu().numpy(), dInv.cpu().numpy(), d[0].cpu().numpy(), d[1].cpu().numpy(),
                    d[2].cpu().numpy(), dinfo.cpu().numpy(), oracle)
    plan.close()


def test_plan_autotune_keeps_a_working_plan(lib, oracle, tmp_path, monkeypatch):
    """The autotuner times chain counts on the caller's buffers and keeps the
    fastest; the plan it keeps gives the reference's results. A second plan of
    the same batch takes the choice from the on-disk cache without timing."""
    monkeypatch.setenv("NPPB_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    torch = pytest.importorskip("torch")
    sys = workloads.uneven_batch(seed=14, count=300, n_lo=2, n_hi=300)
    plan = Plan(sys, FLAGS)
    dev = torch.device("cuda:0")
    cnt = len(sys["n"])
    dA = torch.from_numpy(sys["A"]).to(dev)
    dB = torch.from_numpy(sys["B"]).to(dev)
    dX = torch.zeros_like(dB)
    dInv = torch.zeros(max(plan.inv_elems, 1), dtype=torch.float64, device=dev)
    d = [torch.zeros(cnt, dtype=torch.float64, device=dev) for _ in range(3)]
    dinfo = torch.zeros(cnt, dtype=torch.int32, device=dev)
    chains, lookahead, ms = plan.autotune(dA, dB, dX, dInv, d[0], d[1], d[2], dinfo)
    assert chains in (1, 2, 3, 4, 6) and ms > 0
    dX.zero_()
    plan.execute(dA, dB, dX, dInv, d[0], d[1], d[2], dinfo)
    torch.cuda.synchronize()
    check_vs_oracle(sys, dX.cpu().numpy(), dInv.cpu().numpy(), d[0].cpu().numpy(), d[1].cpu().numpy(),
                    d[2].cpu().numpy(), dinfo.cpu().numpy(), oracle)
    plan.close()
    lines = (tmp_path / "autotune.txt").read_text().splitlines()
    assert len(lines) == 1
    plan2 = Plan(sys, FLAGS)
    dX.zero_()
    c2, la2, ms2 = plan2.autotune(dA, dB, dX, dInv, d[0], d[1], d[2], dinfo)
    assert (c2, la2) == (chains, lookahead) and ms2 == pytest.approx(ms, rel=1e-5)
    assert len((tmp_path / "autotune.txt").read_text().splitlines()) == 1  # a hit appends nothing
    torch.cuda.synchronize()
    check_vs_oracle(sys, dX.cpu().numpy(), dInv.cpu().numpy(), d[0].cpu().numpy(), d[1].cpu().numpy(),
                    d[2].cpu().numpy(), dinfo.cpu().numpy(), oracle)
    plan2.close()


def test_full_uneven_batch_properties(lib):
    """8192 systems, n log-uniform in [4, 512], nrhs in {1, 8, 32}, inverse for 10%."""
    sys = workloads.uneven_batch(seed=2025)
    X, Inv, Det, Sign, Logabs, info = solve_grouped(sys, FLAGS)
    assert not info.any()
    rng = np.random.default_rng(0)
    sample = rng.choice(len(sys["n"]), 160, replace=False)
    for i in sample:
        n, k = int(sys["n"][i]), int(sys["nrhs"][i])
        A = sys["A"][sys["a_off"][i]:sys["a_off"][i] + n * n].reshape(n, n)
        B = sys["B"][sys["b_off"][i]:sys["b_off"][i] + n * k].reshape(n, k)
        x = X[sys["b_off"][i]:sys["b_off"][i] + n * k].reshape(n, k)
        eta = np.abs(B - A @ x).max() / (np.abs(A).sum(1).max() * np.abs(x).max() + np.abs(B).max())
        assert eta < 1e-14, (i, n, eta)
        s, l = np.linalg.slogdet(A)
        assert Sign[i] == s and abs(Logabs[i] - l) <= 1e-12 * abs(l)
        if sys["inv_off"][i] >= 0:
            o = sys["inv_off"][i]
            R = A @ Inv[o:o + n * n].reshape(n, n) - np.eye(n)
            assert np.abs(R).max() < 1e-12


def test_pipelined_host_execution(lib, oracle):
    """Host-buffer execution of a packed batch of >= 512 systems runs as chunks
    whose copies overlap compute; results must match the oracle as before."""
    sys = workloads.uneven_batch(seed=14, count=700, n_lo=1, n_hi=200, nrhs_choices=(1, 4))
    plan = Plan(sys, FLAGS)
    cnt = len(sys["n"])
    for _ in range(2):
        X = np.zeros_like(sys["B"])
        Inv = np.zeros(max(plan.inv_elems, 1))
        Det, Sign, Logabs = np.zeros(cnt), np.zeros(cnt), np.zeros(cnt)
        info = np.full(cnt, -1, np.int32)
        plan.execute_host(sys["A"], sys["B"], X, Inv, Det, Sign, Logabs, info)
        check_vs_oracle(sys, X, Inv, Det, Sign, Logabs, info, oracle)
    plan.close()
