"""Benchmark of the B200 batched dense linear-solve path.

Workload (default, one step): the uneven FP64 batch — 8192 systems, order n
log-uniform in [4, 512], nrhs uniform from {1, 8, 32}, A = N(0,1) + n I, b =
N(0,1) from default_rng (PCG64, the reference's generator); solve and slogdet
for every system, inverse for a seeded 10%. One step = one replay of the plan
(one CUDA graph: a warp-kernel launch per class of orders <= 32, a chain of
step launches per class above, on parallel graph branches) over the whole
batch with inputs already resident in HBM (1.8 GB of matrices: larger than
L2, so no flush is needed between steps).

Arms:
  python bench.py [--gpus N --steps K --warmup W]      this path (one rank per GPU)
  python bench.py --impl reference ...                  the reference's own CPU path
                                                        (oracle/_ref) on the host cores

Prints one JSON line (rank 0). Under torchrun every rank runs its own batch
(seed + rank): weak scaling, no collective on the data path; the step time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched solves/s at ≤1e-10 backward err, refined mixed vs FP64 LU; p50/p99 ms"
WORKLOAD = ("uneven FP64 batch: 8192 systems, n log-uniform [4,512], nrhs {1,8,32}, A=N(0,1)+nI, "
            "solve+slogdet all, inv 10%")
SEED = 2025
KERNEL_NAMES = {"warp_lu": "k_lu_warp", "panel": "k_panel", "update": "k_update", "back": "k_back"}
# what holds each kernel kind below the FP64 ceiling (DMMA and DFMA share it on B200)
LIMITER = {"warp_lu": "latency (one warp per system)", "panel": "latency (one barrier per column)",
           "update": "HBM traffic and latency", "back": "latency (dependent windows)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--count", type=int, default=8192)
    p.add_argument("--cpu-sample", type=int, default=0,
                   help="systems in the CPU baseline's sample (0: the whole batch)")
    p.add_argument("--cpu-sample-1t", type=int, default=256,
                   help="systems in the single-threaded CPU baseline's sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the side measurements (mixed vs FP64, small batch, serving)")
    p.add_argument("--serve-seconds", type=float, default=60.0,
                   help="arrival window of the sustained serving rate (the other rates get 5 s)")
    p.add_argument("--orders", type=int, nargs=2, metavar=("LO", "HI"), default=None,
                   help="profiling aid: only the systems of the batch with LO <= n <= HI")
    p.add_argument("--no-autotune", action="store_true",
                   help="profiling aid: keep the plan's chain count (NPPB_CHAINS) instead of tuning it")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


def fp64_peak_tflops(torch, dev):
    """cuBLAS DGEMM 8192^3 (best of 5) as the measured FP64 tensor-pipe peak."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# Side measurements (rank 0, one GPU): the other workloads of the path, each
# timed with CUDA events on the launching stream after warm-up.

def _event_ms(torch, fn, reps=3, warm=2):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def _berr(torch, A, B, X):
    """max over systems of ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf), on the device."""
    R = B - A @ X
    eta = R.abs().amax((1, 2)) / (A.abs().sum(2).amax(1) * X.abs().amax((1, 2)) + B.abs().amax((1, 2)))
    return float(eta.max().item())


def _orthogonal_pairs(torch, dev, count, n, seed):
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    q1 = torch.linalg.qr(torch.randn(count, n, n, dtype=torch.float64, device=dev, generator=g))[0]
    q2 = torch.linalg.qr(torch.randn(count, n, n, dtype=torch.float64, device=dev, generator=g))[0]
    xt = torch.randn(count, n, 1, dtype=torch.float64, device=dev, generator=g)
    return q1, q2, xt, g


def mixed_vs_fp64(torch, dev, L, _lib):
    """C3 (64 x 1024 and 8 x 4096, kappa 1e2..1e8, mixed FP32 factors) and C4
    (512 x 256, nrhs 4, rows scaled 10^U(-6,6), BF16 factors + equilibration):
    batched solves/s of the refined mixed solve vs the FP64 LU, both to a
    normwise backward error <= 1e-10."""
    P = _lib.ptr
    st = torch.cuda.current_stream().cuda_stream
    out = []
    cases = [(64, 1024, (1e2, 1e4, 1e6, 1e8), 1, 0.0, ("3xtf32",)),
             (8, 4096, (1e2, 1e4, 1e6, 1e8), 1, 0.0, ("3xtf32",)),
             (512, 256, (1e1, 1e3, 1e4), 4, 6.0, ("bf16", "3xtf32"))]
    flag = {"3xtf32": 0, "fp32": _lib.MIXED_FP32_FMA, "tf32": _lib.MIXED_TF32, "bf16": _lib.MIXED_BF16}
    for count, n, kappas, nrhs, decades, factors in cases:
        q1, q2, xt1, g = _orthogonal_pairs(torch, dev, count, n, seed=n)
        xt = xt1.expand(count, n, nrhs).contiguous() if nrhs == 1 else torch.randn(
            count, n, nrhs, dtype=torch.float64, device=dev, generator=g)
        scale = None
        if decades:
            scale = 10.0 ** (torch.rand(count, n, 1, dtype=torch.float64, device=dev, generator=g) * 2 * decades
                             - decades)
        for kappa in kappas:
            sig = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device=dev)
            A = (q1 * sig) @ q2.transpose(1, 2)
            if scale is not None:
                A = A * scale
            A = A.contiguous()
            B = (A @ xt).contiguous()
            X64 = torch.zeros_like(B)
            info = torch.zeros(count, dtype=torch.int32, device=dev)

            def fp64():
                rc = L.nppb_d_linalg_batched(count, n, nrhs, _lib.WANT_SOLVE, P(A), P(B), P(X64), None, None, None,
                                             None, None, None, P(info), st)
                assert rc == 0, _lib.last_error()

            t64 = _event_ms(torch, fp64)
            b64 = _berr(torch, A, B, X64)
            for fac in factors:
                X = torch.zeros_like(B)
                be = torch.zeros(count, dtype=torch.float64, device=dev)
                fe = torch.zeros_like(be)
                it = torch.zeros(count, dtype=torch.int32, device=dev)
                fb = torch.zeros_like(it)

                def mixed():
                    rc = L.nppb_d_solve_mixed_batched(count, n, nrhs, P(A), P(B), P(X), P(xt), 1e-10, 30, flag[fac],
                                                      P(info), P(be), P(fe), P(it), P(fb), st)
                    assert rc == 0, _lib.last_error()

                tm = _event_ms(torch, mixed)
                out.append({
                    "count": count, "n": n, "nrhs": nrhs, "kappa": kappa, "row_scale_decades": decades,
                    "fp64_solves_s": count / (t64 * 1e-3), "fp64_ms": t64, "fp64_max_berr": b64,
                    "mixed_factor": fac, "mixed_solves_s": count / (tm * 1e-3), "mixed_ms": tm,
                    "mixed_over_fp64": t64 / tm, "mixed_max_berr": float(be.max().item()),
                    "mixed_mean_corrections": float(it.float().mean().item()),
                    "mixed_fp64_fallbacks": int(fb.sum().item()), "mixed_max_ferr": float(fe.max().item())})
            del A, B, X64
        del q1, q2
        torch.cuda.empty_cache()
    return out


def mixed_summary(rows):
    """One short entry per (workload, kappa, factor): solves/s ratio over the
    FP64 LU, FP64 fallbacks, worst backward error."""
    if not isinstance(rows, list):
        return rows
    out = []
    for r in rows:
        out.append([f"{r['count']}x{r['n']}" + ("rs" if r.get("row_scale_decades") else ""), r["kappa"],
                    r["mixed_factor"], round(r["mixed_over_fp64"], 3), r["mixed_fp64_fallbacks"],
                    float("%.2g" % r["mixed_max_berr"])])
    return {"columns": ["batch", "kappa", "factor", "mixed_over_fp64", "fp64_fallbacks", "max_berr"],
            "rows": out}


def small_uniform(torch, dev, L, _lib, workloads):
    """C1: (256, 32, 32) + 32 I, solve + det, one launch of the warp kernel."""
    P = _lib.ptr
    A, B = workloads.uniform_batch(seed=SEED)
    dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
    dX = torch.zeros_like(dB)
    det = torch.zeros(256, dtype=torch.float64, device=dev)
    info = torch.zeros(256, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream().cuda_stream

    def run():
        rc = L.nppb_d_linalg_batched(256, 32, 1, _lib.WANT_SOLVE | _lib.WANT_DET, P(dA), P(dB), P(dX), None, P(det),
                                     None, None, None, None, P(info), st)
        assert rc == 0

    ms = _event_ms(torch, run, reps=50, warm=5)
    hX, hdet, hinfo = np.zeros_like(B), np.zeros(256), np.zeros(256, np.int32)
    for _ in range(5):
        L.nppb_solve_det_batched(256, 32, 1, P(A), P(B), P(hX), P(hdet), P(hinfo))
    t0 = time.perf_counter()
    for _ in range(50):
        L.nppb_solve_det_batched(256, 32, 1, P(A), P(B), P(hX), P(hdet), P(hinfo))
    e2e_ms = (time.perf_counter() - t0) / 50 * 1e3
    return {"workload": "256 x 32 x 32 + 32 I, solve + det", "device_us": ms * 1e3,
            "solves_s": 256 / (ms * 1e-3), "e2e_us": e2e_ms * 1e3, "e2e_solves_s": 256 / (e2e_ms * 1e-3),
            "e2e_path": "nppb_solve_det_batched (host buffers, pageable)"}


def gemm_reference_gpu_baseline(torch, dev, L, _lib):
    """Row a10 head-to-head on this B200: the reference's own GPU GEMM (NumPP's
    src/backend/cuda_backend.cu, compiled unmodified for sm_100a: its GpuVTable
    gemm slot, host buffers, 16 x 16 SIMT tiles) against nppb_gemm (host
    buffers, FP64 DMMA) on the same FP64 operands, both through their
    host-buffer calls (copies included); and nppb_d_gemm on device-resident
    operands (CUDA events). A baseline, like cpu_baseline."""
    from oracle.oracle import load_refcuda
    R = load_refcuda()
    if R is None or R.ref_cuda_available() != 1:
        return {"unavailable": "oracle/_ref/refcuda (the reference's CUDA backend) not built or no device"}
    P = _lib.ptr
    out = []
    for n in (1024, 4096):
        rng = np.random.default_rng(n)
        A = rng.standard_normal((n, n))
        B = rng.standard_normal((n, n))
        C = np.zeros((n, n))
        flops = 2.0 * n ** 3

        def host_ms(fn, reps):
            fn()
            t0 = time.perf_counter()
            for _ in range(reps):
                fn()
            return (time.perf_counter() - t0) / reps * 1e3

        reps = 5 if n <= 1024 else 2
        t_ref = host_ms(lambda: R.ref_cuda_gemm(0, n, n, n, A.ctypes.data, B.ctypes.data, C.ctypes.data), reps)
        t_ours = host_ms(lambda: L.nppb_gemm(_lib.DT_FLOAT64, n, n, n, A.ctypes.data, B.ctypes.data,
                                             C.ctypes.data), reps)
        dA, dB = torch.from_numpy(A).to(dev), torch.from_numpy(B).to(dev)
        dC = torch.zeros_like(dA)
        st = torch.cuda.current_stream().cuda_stream
        t_dev = _event_ms(torch, lambda: L.nppb_d_gemm(_lib.DT_FLOAT64, n, n, n, P(dA), P(dB), P(dC), st))
        out.append({"m_n_k": n, "reference_host_ms": t_ref, "reference_tflops": flops / t_ref * 1e-9,
                    "nppb_host_ms": t_ours, "nppb_host_tflops": flops / t_ours * 1e-9,
                    "nppb_device_ms": t_dev, "nppb_device_tflops": flops / t_dev * 1e-9,
                    "host_speedup": t_ref / t_ours})
        del dA, dB, dC
    return {"workload": "C = A B, FP64 row-major, A and B N(0,1)", "rows": out,
            "reference": "NumPP src/backend/cuda_backend.cu gemm_impl / k_gemm_tiled, compiled for sm_100a"}


def serving_run(torch, dev, sustained_seconds, rates=((500, 5.0), (2000, None), (5000, 5.0))):
    """C5: Poisson arrivals at each rate against the serving loop (the rate
    with window None runs for `sustained_seconds`, the others for their
    window); n log-uniform
    [16, 2048] from a seeded pool of 48 matrices (kappa log-uniform [1e1, 1e10]),
    nrhs U[1, 64], 30% of requests new right-hand sides on a resident factor.
    A waiter thread collects completions so the arrival clock never blocks;
    inputs and outputs live in pinned host memory. Returns p50 / p99 latency
    (submission to completion) and completed solves/s per rate."""
    import queue

    from numpp_b200.serving import Server

    rng = np.random.default_rng(SEED)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    pool = []
    for _ in range(48):
        n = int(np.floor(np.exp(rng.uniform(np.log(16), np.log(2049)))))
        kappa = 10.0 ** rng.uniform(1, 10)
        q1 = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))[0]
        q2 = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, device=dev, generator=g))[0]
        sig = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device=dev)
        pool.append(((q1 * sig) @ q2.T).cpu().pin_memory().numpy())
    rhs = torch.randn(2048 * 64, dtype=torch.float64).pin_memory().numpy()
    slots = 384
    xring = torch.zeros(slots, 2048 * 64, dtype=torch.float64).pin_memory().numpy()
    results = []
    for rate, window in rates:
        seconds = sustained_seconds if window is None else window
        lat, statuses = [], []
        q = queue.Queue()
        free = threading.Semaphore(slots)
        with Server(budget_bytes=64 << 30, window_us=500.0, max_batch=512) as srv:
            for A in pool:  # warm-up: every pool entry once
                n = A.shape[0]
                rid, _, _ = srv.submit(A, rhs[:n].reshape(n, 1), X=xring[0, :n].reshape(n, 1))
                srv.wait(rid)

            def waiter():
                while True:
                    rid = q.get()
                    if rid is None:
                        return
                    rc, info, l = srv.wait(rid, timeout_s=120.0)
                    lat.append(l)
                    statuses.append(rc)
                    free.release()

            th = threading.Thread(target=waiter)
            th.start()
            resident = []  # (factor id, n)
            t_next = time.perf_counter()
            t_end = t_next + seconds
            n_req = 0
            while True:
                t_next += rng.exponential(1.0 / rate)
                if t_next >= t_end:
                    break
                while True:
                    d = t_next - time.perf_counter()
                    if d <= 0:
                        break
                    if d > 2e-3:
                        time.sleep(d - 1e-3)
                k = int(rng.integers(1, 65))
                free.acquire()
                slot = n_req % slots
                if resident and rng.random() < 0.3:
                    fid, n = resident[int(rng.integers(len(resident)))]
                    rid, _, _ = srv.submit(None, rhs[:n * k].reshape(n, k), X=xring[slot, :n * k].reshape(n, k),
                                           factor=fid)
                else:
                    A = pool[int(rng.integers(len(pool)))]
                    n = A.shape[0]
                    keep = rng.random() < 0.3
                    rid, _, fid = srv.submit(A, rhs[:n * k].reshape(n, k), X=xring[slot, :n * k].reshape(n, k),
                                             keep=keep)
                    if keep:
                        resident.append((fid, n))
                        if len(resident) > 64:
                            srv.release(resident.pop(0)[0])
                q.put(rid)
                n_req += 1
            q.put(None)
            th.join()
            st = srv.stats()
        lat_ms = np.asarray(lat) * 1e3
        ok = int(sum(1 for r in statuses if r == 0))
        results.append({"rate_per_s": rate, "seconds": seconds, "requests": n_req, "completed_ok": ok,
                        "evicted_or_failed": n_req - ok, "solves_s": ok / seconds,
                        "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
                        "batches": st["batches"]})
    return {"workload": "Poisson arrivals, n log-uniform [16,2048] pool of 48, kappa log-uniform [1e1,1e10], "
                        "nrhs U[1,64], 30% re-solves on resident factors, 64 GB budget, FP64 LU",
            "rates": results}

def bench_config(count: int, world: int) -> dict:
    """The workload description both arms print (same dict, same keys)."""
    return {"workload": WORKLOAD, "count": count, "parallelism": f"replicas{world}",
            "l2": "inputs (1.76 GB of A at 8192 systems) larger than L2; no flush"}


def cpu_reference_sample(sys, sample, threads: int, seed: int = 1):
    """Time the reference's CPU path (oracle/_ref) on the workload, or on a
    random sample of `sample` systems of it; returns (solves/s, kind, cores,
    description, seconds)."""
    from numpp_b200 import workloads
    from oracle import load_oracle, load_ref, ref_available

    if sample is None or sample >= len(sys["n"]):
        sub, what = sys, f"all {len(sys['n'])} systems"
    else:
        rng = np.random.default_rng(seed)
        idx = np.sort(rng.choice(len(sys["n"]), sample, replace=False))
        sub, what = workloads.take(sys, idx), f"{sample} of {len(sys['n'])} systems drawn uniformly (seed {seed})"
    if ref_available():
        r = load_ref()
        t0 = time.perf_counter()
        r.solve_grouped(sub, threads=threads)
        dt = time.perf_counter() - t0
        kind, cores = "reference", threads
    else:
        o = load_oracle()
        t0 = time.perf_counter()
        o.solve_grouped(sub)
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
    desc = f"{what}, numpp::linalg::solve + slogdet + inv per system, {cores} thread(s)"
    return len(sub["n"]) / dt, kind, cores, desc, dt


def run_reference(args):
    """The reference's own CPU implementation (oracle/_ref, NumPP's portable LU
    built from its sources) on every system of the same batch each step, the
    systems fanned out over all host threads (NumPP itself is single-threaded).
    ms_per_step is the measured wall time of a step."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from numpp_b200 import workloads
    sys_ = workloads.uneven_batch(seed=SEED, count=args.count)
    threads = os.cpu_count() or 1
    secs = []
    kind, cores, desc = "port", 1, ""
    for i in range(args.warmup + args.steps):
        _, kind, cores, desc, dt = cpu_reference_sample(sys_, None, threads)
        if i >= args.warmup:
            secs.append(dt)
    step_s = float(np.mean(secs))
    value = args.count / step_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (PCG64 default_rng, seed %d + rank)" % SEED,
        "config": bench_config(args.count, world),
        "p50_ms": 1e3 * float(np.percentile(secs, 50)), "p99_ms": 1e3 * float(np.percentile(secs, 99)),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_b200(args):
    import torch
    import torch.distributed as dist

    from numpp_b200 import _lib, replicas, workloads
    from numpp_b200.grouped import Plan

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", torch.cuda.current_device())
    L = _lib.load()
    assert L.nppb_device_available() == 1, _lib.last_error()

    sys_ = workloads.uneven_batch(seed=SEED + rank, count=args.count)
    if args.orders:
        keep = (sys_["n"] >= args.orders[0]) & (sys_["n"] <= args.orders[1])
        sys_ = workloads.packed_batch(SEED + rank, sys_["n"][keep], sys_["nrhs"][keep],
                                      (sys_["inv_off"] >= 0)[keep], shift=True)
    flags = _lib.WANT_SOLVE | _lib.WANT_SLOGDET | _lib.WANT_INV
    plan = Plan(sys_, flags)
    cnt = len(sys_["n"])
    dA = torch.from_numpy(sys_["A"]).to(dev)
    dB = torch.from_numpy(sys_["B"]).to(dev)
    dX = torch.zeros_like(dB)
    dInv = torch.zeros(max(plan.inv_elems, 1), dtype=torch.float64, device=dev)
    dDet = torch.zeros(cnt, dtype=torch.float64, device=dev)
    dSign = torch.zeros_like(dDet)
    dLog = torch.zeros_like(dDet)
    dInfo = torch.zeros(cnt, dtype=torch.int32, device=dev)
    bufs = (dA, dB, dX, dInv, dDet, dSign, dLog, dInfo)
    stream = torch.cuda.Stream()
    # the plan's chain count, tuned on these buffers before anything is timed
    if args.no_autotune:
        chains, lookahead = None, None
    else:
        chains, lookahead, _ = plan.autotune(*bufs, stream=stream)
    nlaunch = plan.launches()

    def step():
        plan.execute(*bufs, stream=stream)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for i in range(args.steps):
                step()
                ev[i + 1].record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    per_step = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
    total_ms = ev[0].elapsed_time(ev[-1])
    if world > 1:
        total_ms = replicas.max_over_ranks(total_ms, device=dev)
        dist.barrier()
    ms_step = total_ms / args.steps
    value = world * cnt / (ms_step * 1e-3)

    # correctness gate on what was just timed: normwise backward error on a sample
    info = dInfo.cpu().numpy()
    X = dX.cpu().numpy()
    rng = np.random.default_rng(rank)
    worst = 0.0
    for i in rng.choice(cnt, 64, replace=False):
        n, k = int(sys_["n"][i]), int(sys_["nrhs"][i])
        A = sys_["A"][sys_["a_off"][i]:sys_["a_off"][i] + n * n].reshape(n, n)
        B = sys_["B"][sys_["b_off"][i]:sys_["b_off"][i] + n * k].reshape(n, k)
        x = X[sys_["b_off"][i]:sys_["b_off"][i] + n * k].reshape(n, k)
        eta = np.abs(B - A @ x).max() / (np.abs(A).sum(1).max() * np.abs(x).max() + np.abs(B).max())
        worst = max(worst, float(eta))
    assert not info.any() and worst <= 1e-10, (int(info.astype(bool).sum()), worst)

    # per-kernel time (CUDA events around every launch, on the launching stream)
    cls = plan.classes()
    # per-kind launch times on a one-chain plan: every launch timed alone, so
    # the split across chains (which only adds launches) does not skew the kinds
    old_chains = os.environ.get("NPPB_CHAINS")
    os.environ["NPPB_CHAINS"] = "1"
    tplan = Plan(sys_, flags)
    if old_chains is None:
        del os.environ["NPPB_CHAINS"]
    else:
        os.environ["NPPB_CHAINS"] = old_chains
    kern = tplan.time_kernels(*bufs, stream=stream)
    tplan.close()
    top = max(kern, key=lambda k: kern[k][0])
    top_ms, flops_top = kern[top]
    peak64 = fp64_peak_tflops(torch, dev)
    achieved = flops_top / (top_ms * 1e-3) / 1e12
    # DRAM bytes per step of the top kernel kind, from the committed one-pass
    # ncu capture of one plan execution (profiles/uneven8192_step_traffic.json)
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "uneven8192_step_traffic.json")
    if os.path.exists(tfile) and args.count == 8192:
        with open(tfile) as f:
            traffic = json.load(f).get("bytes_per_step", {}).get(KERNEL_NAMES[top])

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    hA, hB = pin(sys_["A"]), pin(sys_["B"])
    hX = pin(np.zeros_like(sys_["B"]))
    hInv = pin(np.zeros(max(plan.inv_elems, 1)))
    hDet, hSign, hLog = pin(np.zeros(cnt)), pin(np.zeros(cnt)), pin(np.zeros(cnt))
    hInfo = pin(np.zeros(cnt, np.int32))
    for _ in range(max(1, args.warmup)):
        plan.execute_host(hA, hB, hX, hInv, hDet, hSign, hLog, hInfo)
    if world > 1:
        dist.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        plan.execute_host(hA, hB, hX, hInv, hDet, hSign, hLog, hInfo)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_step = float(np.mean(e2e_ms))
    if world > 1:
        e2e_step = replicas.max_over_ranks(e2e_step, device=dev)
    h2d = 8 * (plan.a_elems + plan.b_elems)
    d2h = 8 * (plan.b_elems + plan.inv_elems + 3 * cnt) + 4 * cnt

    cpu = None
    cpu_1t = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, kind, cores, desc, _ = cpu_reference_sample(sys_, args.cpu_sample or None, os.cpu_count() or 1)
        cpu = {"value": rate, "unit": "solves/s", "cores": cores, "kind": kind, "sample": desc}
        # NumPP as a user calls it: one thread, one system after another
        rate1, kind1, _, desc1, _ = cpu_reference_sample(sys_, args.cpu_sample_1t, 1)
        cpu_1t = {"value": rate1, "unit": "solves/s", "cores": 1, "kind": kind1, "sample": desc1}

    flops_step = workloads.uneven_flops(sys_)
    # The workload's bound is the FP64 tensor pipe (17 flop/B of algorithmic
    # traffic, above the FP64 ridge): achieved = the dominant kind's algorithmic
    # flops over its launch time, against cuBLAS DGEMM measured in this run.
    # The HBM view beside it: the same kind's bytes (each trailing element read
    # and written once per 32-column step) over the same time.
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_view = None
    if top == "update":
        bytes_top = workloads.step_update_bytes(sys_)
        ach_gbs = bytes_top / (top_ms * 1e-3) / 1e9
        hbm_view = {"achieved": ach_gbs, "peak": hbm or 6650.0, "unit": "GB/s", "frac": ach_gbs / (hbm or 6650.0),
                    "peak_source": ("measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs), of measured" if hbm
                                    else "6.65 TB/s, of fallback (no MEASURED_PEAKS.json)"),
                    "bytes_per_step": bytes_top,
                    "algorithmic_min_bytes_whole_step": workloads.uneven_bytes(sys_),
                    "traffic_per_step": traffic,
                    "traffic_source": "ncu one-pass DRAM capture of one plan execution "
                                      "(profiles/uneven8192_step_traffic.json)"}
    roofline = {"bound": "tensor", "kernel": KERNEL_NAMES[top], "limiter": LIMITER[top],
                "achieved": achieved, "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64,
                "peak_source": "measured cuBLAS FP64 GEMM 8192^3 on this GPU (burst), of measured",
                "traffic": traffic, "ms_per_step": top_ms, "flops_per_step": flops_top,
                "whole_step_tflops": flops_step / (ms_step * 1e-3) / 1e12,
                "note": ("k_rows + k_update" if top == "update" else KERNEL_NAMES[top])
                        + " summed over one step's launches on a one-chain copy of the plan, each timed alone",
                **({"hbm_view": hbm_view} if hbm_view else {})}
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        plan.close()
        del bufs, dA, dB, dX, dInv
        torch.cuda.empty_cache()
        # a side measurement that fails is reported, not fatal to the headline line
        for key, fn in (("small_batch", lambda: small_uniform(torch, dev, L, _lib, workloads)),
                        ("gemm_reference_gpu_baseline", lambda: gemm_reference_gpu_baseline(torch, dev, L, _lib)),
                        ("mixed_vs_fp64", lambda: mixed_vs_fp64(torch, dev, L, _lib)),
                        ("serving", lambda: serving_run(torch, dev, args.serve_seconds))):
            try:
                extras[key] = fn()
            except Exception as e:  # noqa: BLE001
                extras[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
        extras["mixed_vs_fp64_summary"] = mixed_summary(extras.get("mixed_vs_fp64"))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (PCG64 default_rng, seed %d + rank)" % SEED,
            "config": {**bench_config(cnt, world), **({"orders_only": list(args.orders)} if args.orders else {})},
            "plan": {"graph": True, "autotuned_chains": chains, "autotuned_lookahead": lookahead,
                     "classes": [f"{c[0]}<= {c[1]}: {c[2]}" for c in cls]},
            "p50_ms": float(np.percentile(per_step, 50)), "p99_ms": float(np.percentile(per_step, 99)),
            "gflops": flops_step * world / (ms_step * 1e-3) / 1e9,
            "max_backward_error_sample": worst,
            "roofline": roofline,
            "kernels": {KERNEL_NAMES[k]: {"ms": round(v[0], 4), "tflops": v[1] / max(v[0], 1e-9) / 1e9}
                        for k, v in kern.items()},
            "e2e": {"value": world * cnt / (e2e_step * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step,
                    "path": "nppb_plan_execute_host (C ABI), pinned host buffers"},
            "gpu_launches": args.steps * nlaunch,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "cpu_baseline_1thread": cpu_1t,
            "hbm_peak_gbs": hbm,
            **extras,
        }
        # the compact mixed-vs-FP64 figures last: the end of the line is what log tails keep
        if "mixed_vs_fp64_summary" in line:
            line["mixed_vs_fp64_summary"] = line.pop("mixed_vs_fp64_summary")
        print(json.dumps(line), flush=True)
    plan.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
