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


def _shard_worker(rank, world, port, out):
    """One rank of a scene-sharded batch pass: its round-robin share of the scenes as a
    batch of its own through the oracle, results gathered to every rank over gloo."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world)
    try:
        from oracle import oracle as o
        from untangling26_b200 import synthetic
        full = synthetic.batch_scenes(num=5, seed=11, tris_lo=2000, tris_hi=3000)
        ids = multirank.scene_shard(full.meta["num"], rank, world)
        sub = synthetic.sub_batch(full, ids)
        ef, idx = o.detect_ef(sub)
        run = o.PrpRun(sub, ef, idx, o.prp_params(max_contours=1 << 20, batch_size=1 << 20))
        mine = {}
        for j, s in enumerate(ids):
            cs = [c for c in range(len(run.contours)) if run.results[c]["object_id0"] // 2 == j]
            mine[s] = [(run.results[c].tobytes(), run.hits[c]["type"].tobytes(), run.hits[c]["bary"].tobytes(),
                        run.hits[c]["dist"].tobytes()) for c in cs]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, gathered))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_scene_shards_cover_the_batch():
    """The union of the two ranks' shard passes equals the single-rank pass of the whole
    batch, scene by scene (every result field but the batch positions; the supports' types,
    barycentres and depths)."""
    import numpy as np

    from oracle import oracle as o
    from untangling26_b200 import synthetic
    o.build()
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_shard_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    union = {}
    for part in res[0]:
        union.update(part)
    assert res[0] == res[1] and sorted(union) == list(range(5))
    full = synthetic.batch_scenes(num=5, seed=11, tris_lo=2000, tris_hi=3000)
    ef, idx = o.detect_ef(full)
    run = o.PrpRun(full, ef, idx, o.prp_params(max_contours=1 << 20, batch_size=1 << 20))
    skip = ("contour_idx", "object_id0", "object_id1")
    assert len(run.contours) > 0
    for s in range(5):
        cs = [c for c in range(len(run.contours)) if run.results[c]["object_id0"] // 2 == s]
        assert len(cs) == len(union[s])
        for c, (rb, ht, hb, hd) in zip(cs, union[s]):
            r = np.frombuffer(rb, dtype=run.results.dtype)[0]
            for name in run.results.dtype.names:
                if name not in skip:
                    assert np.array_equal(r[name], run.results[c][name]), (s, name)
            assert ht == run.hits[c]["type"].tobytes() and hb == run.hits[c]["bary"].tobytes() and hd == run.hits[c]["dist"].tobytes()
