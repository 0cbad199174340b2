"""Multi-GPU plumbing for the assembly path: one process per GPU, no
collective in the data path.

The path shards only as independent units (batched specimens, or one
specimen per rank).  Each rank assembles its own share on its own GPU;
the only communication is the timing, reduced as the maximum over ranks, and
the counts, summed, after the timed region.  Ranks take specimens
round-robin, so uneven specimen sizes spread evenly enough without a
partitioner."""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Items of this rank: rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, n_items, world))


def reduce_max(values, device=None):
    """Element-wise maximum over ranks of a list of floats (identity without
    an initialised process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


def reduce_sum(values, device=None):
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().tolist()
