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

Or the splats are sharded (``render_sharded``): each rank holds a contiguous
share of the scene, projects it for the whole frame, and sends every
projected splat to the owners of the row windows its bbox meets (one
all-to-all of counts, one of records); each owner bins, sorts and blends its
window from the records it received, and the windows are gathered. The frame
equals the one-device render of the whole scene bit for bit.
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


def shard_range(n: int, rank: int, world: int):
    """[s0, s1): rank `rank`'s contiguous share of n splats (shards in scene
    order, sizes differing by one at most)."""
    return n * rank // world, n * (rank + 1) // world


def exchange_records(send, counts, record_bytes: int, world: int):
    """The all-to-all of the sharded frame: `send` (a uint8 tensor) holds this
    rank's records for window 0, then window 1, ... (counts[k] records of
    record_bytes bytes for window k, whose owner is rank k); returns the
    records this rank's window receives, the senders' runs concatenated in
    rank order (so in scene order), and their count. One all-to-all of the
    counts, one of the records (NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist

    if world <= 1 or not (dist.is_available() and dist.is_initialized()):
        return send, int(counts[0])
    dev = send.device
    cnt = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=dev)
    rcnt = torch.empty_like(cnt)
    dist.all_to_all_single(rcnt, cnt)
    rcounts = [int(c) for c in rcnt.tolist()]
    recv = torch.empty(sum(rcounts) * record_bytes, dtype=torch.uint8, device=dev)
    dist.all_to_all_single(recv, send, [c * record_bytes for c in rcounts],
                           [int(c) * record_bytes for c in counts])
    return recv, sum(rcounts)


def gather_rows(part, wins, width: int, rank: int, world: int):
    """Every rank's row window (part: this rank's (rows, width, 3) uint8
    tensor) assembled into the whole (height, width, 3) frame on every rank
    (one all_gather of equal-size padded windows); a numpy array."""
    import numpy as np
    import torch
    import torch.distributed as dist

    height = wins[-1][0] + wins[-1][1]
    if world <= 1 or not (dist.is_available() and dist.is_initialized()):
        return part.cpu().numpy()
    most = max(n for _, n in wins)
    pad = torch.zeros((most, width, 3), dtype=torch.uint8, device=part.device)
    pad[:part.shape[0]] = part
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    frame = np.empty((height, width, 3), np.uint8)
    for (r0, n), p in zip(wins, parts):
        if n:
            frame[r0:r0 + n] = p[:n].cpu().numpy()
    return frame


def render_sharded(shard_records, render_records, width: int, height: int, rank: int, world: int,
                   record_bytes: int, tile: int = 16):
    """One frame from splats sharded over the ranks of the process group.

    shard_records(bounds) -> (send, counts): this rank's records for the row
    windows [bounds[k], bounds[k + 1]) (``CudaRenderer.shard_records`` of its
    shard); render_records(records, n, row0, rows) -> (rows, width, 3) uint8
    tensor: the window drawn from received records
    (``CudaRenderer.render_records``). Window k (``row_windows``) belongs to
    rank k. Returns the whole frame (numpy) on every rank."""
    wins = row_windows(height, world, tile)
    bounds = [r0 for r0, _ in wins] + [height]
    send, counts = shard_records(bounds)
    recv, n = exchange_records(send, counts, record_bytes, world)
    row0, rows = wins[rank]
    part = render_records(recv, n, row0, rows)
    return gather_rows(part, wins, width, rank, world)


def render_sharded_frame(renderer, view, width: int, height: int, background, rank: int, world: int):
    """``render_sharded`` with a CudaRenderer holding this rank's shard (a
    contiguous share of the scene, shards in rank order). The records and
    windows cross over NCCL on the renderer's device, or through host memory
    when the process group is gloo. Returns (frame, visible splats of this
    shard, (splat, tile) pairs of this rank's window)."""
    import torch
    import torch.distributed as dist

    from . import _native as N

    dev = torch.device(f"cuda:{renderer.device}")
    via_host = world > 1 and dist.is_available() and dist.is_initialized() and dist.get_backend() == "gloo"
    info = {}

    def shard(bounds):
        send, counts, info["visible"] = renderer.shard_records(view, width, height, bounds)
        return (send.cpu() if via_host else send), counts

    def draw(records, n, row0, rows):
        out = torch.empty((rows, width, 3), dtype=torch.uint8, device=dev)
        if rows:
            _, st = renderer.render_records(view, width, height, background, records.to(dev), row0, rows,
                                            out=out, stats=True)
            info["overlaps"] = st.overlaps
        return out.cpu() if via_host else out

    frame = render_sharded(shard, draw, width, height, rank, world, N.SPLAT_RECORD_BYTES)
    return frame, info.get("visible", 0), info.get("overlaps", 0)
