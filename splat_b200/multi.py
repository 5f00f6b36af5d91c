"""View-parallel rendering over several GPUs, one process per GPU.

The reference draws one view per ``Renderer::render`` call; frames and batch
views are independent units, so N ranks each render a disjoint share of the
views with no collective on the data path. The only collectives are the
timing ones: a barrier around the timed region and the maximum of the ranks'
device times (NCCL on GPUs; the same calls run over gloo on CPU in tests).
"""

from __future__ import annotations

import os


def dist_env():
    """(rank, world size, local rank) from torchrun's environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def shard(items, rank: int, world: int) -> list:
    """Rank `rank`'s share of `items`: every world-th item from `rank` (the
    shares of all ranks are disjoint and cover the list; an empty share
    falls back to the whole list so that every rank has work)."""
    items = list(items)
    if world <= 1:
        return items
    mine = items[rank::world]
    return mine if mine else items


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the job's time is its slowest
    rank's); the value itself when no process group is initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, seconds_per_rank: float, world: int, device=None) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / max_over_ranks(seconds_per_rank, device)
