"""Multi-GPU plumbing for the batched solve: replicas only.

Systems are independent, so a batch shards across ranks by contiguous slices
of systems with no exchange on the data path (the reference has no parallel
path at all: src/linalg/batched.cpp:51-108 loops one matrix at a time). One
process per GPU over torch.distributed; the only collectives are the
max-over-ranks of a timing and, when a caller wants every result on one rank,
a gather of the per-rank outputs.
"""
from __future__ import annotations

import numpy as np

from . import workloads


def shard_bounds(count: int, world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of the systems rank `rank` owns: contiguous, sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world or count < 0:
        raise ValueError("need world > 0, 0 <= rank < world, count >= 0")
    base, extra = divmod(count, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard(sys: dict, world: int, rank: int) -> dict:
    """This rank's systems of a packed batch, repacked (offsets from zero)."""
    lo, hi = shard_bounds(len(sys["n"]), world, rank)
    return workloads.take(sys, np.arange(lo, hi))


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (a step time: the job is as slow as its slowest rank)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(local: np.ndarray):
    """Concatenation of every rank's 1-D array in rank order on rank 0 (None elsewhere)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return local
    parts = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(np.ascontiguousarray(local), parts, dst=0)
    return np.concatenate(parts) if dist.get_rank() == 0 else None
