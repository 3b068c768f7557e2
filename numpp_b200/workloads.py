"""Seeded synthetic inputs for the batched solve workloads.

numpy's ``default_rng(seed)`` (PCG64 + ziggurat normals) is the generator NumPP
reproduces bit-for-bit as ``numpp::random::default_rng`` (src/random/*,
pinned by NumPP's tests/test_rng_bitexact.cpp:12-19), so these arrays are the
inputs the reference itself would draw with the same seed and draw order.

Packed (uneven) layout, used by ``Plan`` and the grouped C ABI: every matrix
row-major back to back in one float64 array (``a_off``), right-hand sides /
solutions back to back in another (``b_off``), inverses back to back for the
systems that ask for one (``inv_off`` = -1 otherwise).
"""
from __future__ import annotations

import numpy as np


def uniform_batch(seed: int, count: int = 256, n: int = 32, nrhs: int = 1, shift: float | None = None):
    """A = N(0,1) + shift*I (shift defaults to n), then b = N(0,1), from one generator:
    the (256, 32, 32) solve + det workload at the defaults."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((count, n, n))
    A += (float(n) if shift is None else shift) * np.eye(n)
    B = rng.standard_normal((count, n, nrhs))
    return A, B


def uneven_batch(seed: int, count: int = 8192, n_lo: int = 4, n_hi: int = 512,
                 nrhs_choices=(1, 8, 32), inv_fraction: float = 0.1):
    """The uneven FP64 batch: n = floor(exp(U(ln n_lo, ln(n_hi+1)))), nrhs uniform over
    `nrhs_choices`, A = N(0,1) + n*I, b = N(0,1), inverse for a seeded `inv_fraction`.

    Draw order: n (count uniforms), nrhs (count choices), inverse mask (count
    uniforms), then all matrix entries (system order, row-major), then all
    right-hand sides.
    """
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi + 1), size=count))).astype(np.int32)
    n = np.clip(n, n_lo, n_hi)
    nrhs = rng.choice(np.asarray(nrhs_choices, np.int32), size=count).astype(np.int32)
    want_inv = rng.random(count) < inv_fraction
    nn = n.astype(np.int64) ** 2
    nb = n.astype(np.int64) * nrhs
    a_off = np.concatenate([[0], np.cumsum(nn)[:-1]]).astype(np.int64)
    b_off = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    inv_sizes = np.where(want_inv, nn, 0)
    inv_off = np.where(want_inv, np.concatenate([[0], np.cumsum(inv_sizes)[:-1]]), -1).astype(np.int64)
    A = rng.standard_normal(int(nn.sum()))
    # + n*I: diagonal element j of system i sits at a_off[i] + j*(n[i]+1)
    reps = n.astype(np.int64)
    sys_of = np.repeat(np.arange(count), reps)
    j = np.arange(int(reps.sum())) - np.repeat(np.concatenate([[0], np.cumsum(reps)[:-1]]), reps)
    A[a_off[sys_of] + j * (n[sys_of].astype(np.int64) + 1)] += n[sys_of]
    B = rng.standard_normal(int(nb.sum()))
    return {
        "n": n, "nrhs": nrhs, "a_off": a_off, "b_off": b_off, "inv_off": inv_off,
        "A": A, "B": B, "inv_size": int(inv_sizes.sum()), "count": count,
    }


def packed_batch(seed: int, n, nrhs, want_inv, shift: bool = False) -> dict:
    """A packed batch of given orders / right-hand-side counts / inverse mask:
    A = N(0,1) (+ n*I with shift), b = N(0,1), matrices then right-hand sides
    drawn from one generator in system order."""
    rng = np.random.default_rng(seed)
    n = np.asarray(n, np.int32)
    nrhs = np.asarray(nrhs, np.int32)
    want = np.asarray(want_inv, bool)
    nn = n.astype(np.int64) ** 2
    nb = n.astype(np.int64) * nrhs
    a_off = np.concatenate([[0], np.cumsum(nn)[:-1]]).astype(np.int64)
    b_off = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    inv_sizes = np.where(want, nn, 0)
    inv_off = np.where(want, np.concatenate([[0], np.cumsum(inv_sizes)[:-1]]), -1).astype(np.int64)
    A = rng.standard_normal(int(nn.sum()))
    if shift:
        for i, ni in enumerate(n):
            A[a_off[i]:a_off[i] + ni * ni].reshape(ni, ni)[np.diag_indices(ni)] += ni
    B = rng.standard_normal(int(nb.sum()))
    return {"n": n, "nrhs": nrhs, "a_off": a_off, "b_off": b_off, "inv_off": inv_off, "A": A, "B": B,
            "inv_size": int(inv_sizes.sum()), "count": len(n)}


def take(sys: dict, idx) -> dict:
    """Repack a subset of an uneven batch (for bounded CPU samples and parity cases)."""
    idx = np.asarray(idx)
    n = sys["n"][idx]
    k = sys["nrhs"][idx]
    nn = n.astype(np.int64) ** 2
    nb = n.astype(np.int64) * k
    a_off = np.concatenate([[0], np.cumsum(nn)[:-1]]).astype(np.int64)
    b_off = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
    want = sys["inv_off"][idx] >= 0
    inv_sizes = np.where(want, nn, 0)
    inv_off = np.where(want, np.concatenate([[0], np.cumsum(inv_sizes)[:-1]]), -1).astype(np.int64)
    A = np.concatenate([sys["A"][o:o + s] for o, s in zip(sys["a_off"][idx], nn)]) if len(idx) else np.zeros(0)
    B = np.concatenate([sys["B"][o:o + s] for o, s in zip(sys["b_off"][idx], nb)]) if len(idx) else np.zeros(0)
    return {"n": n, "nrhs": k, "a_off": a_off, "b_off": b_off, "inv_off": inv_off, "A": A, "B": B,
            "inv_size": int(inv_sizes.sum()), "count": len(idx)}


def lu_flops(n) -> np.ndarray:
    """LAPACK getrf flop count 2/3 n^3 - 1/2 n^2 + 5/6 n."""
    n = np.asarray(n, np.float64)
    return 2.0 / 3.0 * n**3 - 0.5 * n**2 + 5.0 / 6.0 * n


def getrs_flops(n, k) -> np.ndarray:
    n = np.asarray(n, np.float64)
    return 2.0 * n**2 * np.asarray(k, np.float64) - n * np.asarray(k, np.float64)


def uneven_flops(sys: dict) -> float:
    """Algorithmic flops of solve + slogdet (one shared getrf) + inverse (getrf + 4/3 n^3)."""
    n = sys["n"].astype(np.float64)
    inv = sys["inv_off"] >= 0
    return float(lu_flops(n).sum() + getrs_flops(n, sys["nrhs"]).sum() + (4.0 / 3.0 * n[inv] ** 3).sum())


def uneven_bytes(sys: dict) -> float:
    """Algorithmic minimum bytes: read A and b once, write x, inverses, sign/logdet/info."""
    nn = sys["n"].astype(np.float64) ** 2
    nb = sys["n"].astype(np.float64) * sys["nrhs"]
    inv = sys["inv_off"] >= 0
    return float(8 * nn.sum() + 16 * nb.sum() + 8 * nn[inv].sum() + 20 * len(nn))


def step_update_bytes(sys: dict, nb: int = 32) -> float:
    """Algorithmic DRAM bytes of the step-wise trailing updates (row moves + U12
    and A22 -= L21 U12) of one uneven batch, FP64: at each 32-column step of a
    system of order n > 32, every trailing element (matrix columns right of the
    panel, right-hand sides, inverse columns) below the panel is read and
    written once (16 B), L21 is read once per 64-column strip (8 B x 32 per
    row), and the 32 panel rows of those columns are read and written by the
    row-move / U12 pass (16 B each). Orders <= 32 take the warp kernel."""
    total = 0.0
    for n, k, inv in zip(sys["n"].astype(np.int64), sys["nrhs"].astype(np.int64), sys["inv_off"] >= 0):
        if n <= nb:
            continue
        for k0 in range(0, n, nb):
            below = n - k0 - nb
            width = max(below, 0) + k + (n if inv else 0)
            if below > 0:
                total += 16.0 * below * width + 8.0 * below * nb * ((width + 63) // 64)
            total += 16.0 * min(nb, n - k0) * width
    return total


def conditioned_batch(seed: int, count: int, n: int, kappa: float, nrhs: int = 1,
                      row_scale_decades: float = 0.0):
    """A = Q1 diag(sigma) Q2^T with Q from the QR of N(0,1) matrices and sigma
    log-spaced from 1 to kappa; optionally rows scaled by 10^U(-d, d); x_true
    = N(0,1); b = A x_true in FP64. Returns (A, B, X_true)."""
    rng = np.random.default_rng(seed)
    sigma = np.logspace(0.0, np.log10(kappa), n)
    A = np.empty((count, n, n))
    for i in range(count):
        q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
        q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
        A[i] = (q1 * sigma) @ q2.T
    if row_scale_decades:
        A *= 10.0 ** rng.uniform(-row_scale_decades, row_scale_decades, size=(count, n, 1))
    X = rng.standard_normal((count, n, nrhs))
    B = A @ X
    return A, B, X
