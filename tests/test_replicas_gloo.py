"""Replica sharding across ranks, run as two gloo ranks on the CPU: every
system solved exactly once, results gathered in order, timings reduced to the
max over ranks. The per-rank solver here is the oracle (the CPU checker)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from numpp_b200 import replicas, workloads


def test_shard_bounds_cover_every_system_once():
    for count in (0, 1, 7, 8192):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard_bounds(count, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard_bounds(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from oracle import load_oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys_ = workloads.uneven_batch(seed=11, count=21, n_lo=4, n_hi=40)
        mine = replicas.shard(sys_, world, rank)
        X, s, la, inv, ok = load_oracle().solve_grouped(mine)
        gathered = replicas.gather_to_rank0(X)
        slowest = replicas.max_over_ranks(1.0 + rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "X.npy"), gathered)
            np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_solve_disjoint_shards(tmp_path, oracle):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    sys_ = workloads.uneven_batch(seed=11, count=21, n_lo=4, n_hi=40)
    X_all, *_ = oracle.solve_grouped(sys_)
    assert np.array_equal(np.load(tmp_path / "X.npy"), X_all)
    assert float(np.load(tmp_path / "slowest.npy")[0]) == 2.0
