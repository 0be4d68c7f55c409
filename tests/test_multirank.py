"""Rank plumbing of one-process-per-GPU runs, on CPU with the gloo backend (world size 2):
scene sharding covers every scene once, and the job time is the maximum over ranks on every
rank."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from untangling26_b200 import multirank


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
    try:
        ws, r, local = multirank.dist_env()
        assert (ws, r, local) == (world, rank, rank)
        local_ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        t = multirank.job_time_ms(local_ms)
        shard = multirank.scene_shard(7, rank, world)
        out.put((rank, t, shard, multirank.job_throughput(100, world, t)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_shards():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [t for _, t, _, _ in res] == [20.0, 20.0]  # the max over ranks, seen by both
    shards = [s for _, _, s, _ in res]
    assert sorted(shards[0] + shards[1]) == list(range(7)) and not set(shards[0]) & set(shards[1])
    assert res[0][3] == pytest.approx(100 * 2 / 0.020)


def test_single_process_defaults():
    assert multirank.dist_env({}) == (1, 0, 0)
    assert multirank.job_time_ms(12.5) == 12.5
    assert multirank.scene_shard(5, 0, 1) == [0, 1, 2, 3, 4]
    with pytest.raises(ValueError):
        multirank.scene_shard(5, 2, 2)
