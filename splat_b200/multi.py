"""Rendering over several GPUs, one process per GPU.

The reference draws one view per ``Renderer::render`` call; frames and batch
views are independent units, so N ranks each render a disjoint share of the
views with no collective on the data path. The only collectives are the
timing ones: a barrier around the timed region and the maximum of the ranks'
device times (NCCL on GPUs; the same calls run over gloo on CPU in tests).

One frame can also be split by rows: each rank holds the scene, renders a
window of whole tile rows (``CudaRenderer.render_rows``: the projection is
repeated per rank, the binning, sorts and blend are shared out) and the
windows are gathered (``render_split``).
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


def row_windows(height: int, world: int, tile: int = 16) -> list:
    """(row0, rows) per rank: the frame's tile rows shared out as evenly as
    whole tile rows allow, in order, covering [0, height) disjointly (a rank
    may get 0 rows when there are fewer tile rows than ranks)."""
    tiles = (height + tile - 1) // tile
    out, t0 = [], 0
    for r in range(world):
        t1 = t0 + tiles // world + (1 if r < tiles % world else 0)
        row0, row1 = min(t0 * tile, height), min(t1 * tile, height)
        out.append((row0, row1 - row0))
        t0 = t1
    return out


def render_split(render_rows, width: int, height: int, rank: int, world: int, tile: int = 16, device=None):
    """One frame over the ranks of the process group: this rank draws its
    row window with ``render_rows(row0, rows) -> (rows, width, 3) u8 array``
    and every rank receives the whole (height, width, 3) frame (one
    all_gather of equal-size padded windows). Without a process group (or one
    rank) the frame is drawn in one window."""
    import numpy as np
    import torch
    import torch.distributed as dist

    if world <= 1 or not (dist.is_available() and dist.is_initialized()):
        return render_rows(0, height)
    wins = row_windows(height, world, tile)
    row0, rows = wins[rank]
    most = max(n for _, n in wins)
    part = np.zeros((most, width, 3), np.uint8)
    if rows:
        part[:rows] = render_rows(row0, rows)
    t = torch.from_numpy(part).to(device) if device is not None else torch.from_numpy(part)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    frame = np.empty((height, width, 3), np.uint8)
    for (r0, n), p in zip(wins, parts):
        if n:
            frame[r0:r0 + n] = p[:n].cpu().numpy()
    return frame
