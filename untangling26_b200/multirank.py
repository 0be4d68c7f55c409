"""Rank plumbing for one-process-per-GPU runs of the untangling pass.

The pass shards by independent scenes (a scene is an object set that touches no other scene), so
ranks exchange no data on the path: each rank runs its own scenes and only the step timing is
combined, as the maximum over ranks. These helpers work with any torch.distributed backend
(NCCL on GPUs, gloo on CPU).
"""
import torch


def dist_env(environ=None):
    """(world_size, rank, local_rank) from torchrun's environment (1, 0, 0 when absent)."""
    import os
    env = os.environ if environ is None else environ
    return int(env.get("WORLD_SIZE", "1")), int(env.get("RANK", "0")), int(env.get("LOCAL_RANK", "0"))


def scene_shard(num_scenes, rank, world):
    """Scene ids a rank owns when a batch of independent scenes is split across ranks
    (round robin, so sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, num_scenes, world))


def job_time_ms(local_ms, device=None):
    """The job's time: the maximum of the ranks' times (every rank gets it)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank, world, job_ms):
    """Whole-job throughput: the units all ranks processed over the job time."""
    return units_per_rank * world / (job_ms / 1e3)
