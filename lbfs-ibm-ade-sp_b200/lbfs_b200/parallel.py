"""Multi-GPU plumbing: one process per GPU, torch.distributed for control.

The step has no exchange between independent instances (replicas of one
workload, or the members of an ensemble), so the data path carries no
collective: ranks only agree on timing (max over ranks) and gather per-instance
metrics at the end.  Works with the NCCL backend on GPUs and with gloo on CPU.
"""
import os

__all__ = ["dist_env", "shard_instances", "max_over_ranks", "gather_objects"]


def dist_env():
    """(rank, local_rank, world_size) from the torchrun environment (1 process when absent)."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def shard_instances(costs, world):
    """Deterministic longest-processing-time assignment of independent instances
    to ranks: instances by decreasing cost (ties by index) each go to the rank
    with the least total so far (ties by rank).  Returns one sorted index list
    per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += costs[i]
    return [sorted(s) for s in shards]


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (the value itself with one process)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_objects(obj):
    """List of every rank's object, in rank order, on every rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
