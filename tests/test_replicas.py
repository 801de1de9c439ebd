"""Replica plumbing of multi-GPU runs, exercised as two gloo ranks on CPU:
disjoint query shards, max-over-ranks timing and whole-job throughput."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from nigiri_b200 import replicas


def test_shards_partition_the_stream():
    for n in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            covered = [i for p in parts for i in p]
            assert covered == list(range(n))
            assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def test_seeds_differ_per_rank():
    seeds = {replicas.query_seed(1002, r) for r in range(8)}
    assert len(seeds) == 8


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        # rank r pretends to have taken (r + 1) seconds of device time and
        # 2 (r + 1) seconds of wall time for its 1024 queries
        times = replicas.max_over_ranks([rank + 1.0, 2.0 * (rank + 1)], dist)
        qps = replicas.whole_job_throughput(1024, world, times[0])
        shape = replicas.from_rank0([32 + rank, 256, 8 * (rank + 1), 2, 4, rank], dist)
        dist.barrier()
        out[rank] = (times, qps, list(replicas.shard(4096, rank, world)), shape)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    assert set(out.keys()) == {0, 1}
    for r in range(world):
        times, qps, part, shape = out[r]
        assert times == [2.0, 4.0]          # max over ranks, on every rank
        assert shape == [32, 256, 8, 2, 4, 0]  # rank 0's launch shape, on every rank
        assert qps == pytest.approx(1024 * 2 / 2.0)
    assert sorted(out[0][2] + out[1][2]) == list(range(4096))
