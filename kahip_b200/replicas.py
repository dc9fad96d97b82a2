"""Host logic of the multi-GPU replica form: one process per GPU, every rank
partitions its own items (graphs, seeds or replicas of one graph) with no
collective on the data path; the only collectives are the timing reduction
(max over ranks) and barriers around the timed region.

Works with any torch.distributed backend (nccl on GPUs, gloo on CPU)."""
from __future__ import annotations

import os


def rank_env() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def member_seed(seed: int, rank: int, world: int) -> int:
    """Seed of a rank's population member: seed * size + rank, as KaFFPaE
    gives each of its processes (lib/parallel_mh/parallel_mh_async.cpp:54)."""
    return seed * world + rank


def shard_items(sizes, rank: int, world: int) -> list[int]:
    """Indices of the items this rank partitions: items in decreasing size
    order (ties by index) are dealt to the rank with the least work so far
    (ties to the smaller rank).  Every rank computes the same assignment from
    the same sizes, so no communication is needed."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += sizes[i]
        if r == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over all ranks (the rank's own value when not
    distributed)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
