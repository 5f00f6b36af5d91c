"""The view-parallel path with two ranks on CPU (gloo): disjoint shares that
cover the views, the maximum of the ranks' times on every rank, the
whole-job rate."""

import os
import socket

import pytest
import torch.multiprocessing as mp

from splat_b200 import multi


def test_shard_covers_disjointly():
    views = list(range(40))
    for world in (1, 2, 3, 4, 8):
        shares = [multi.shard(views, r, world) for r in range(world)]
        flat = sorted(v for s in shares for v in s)
        assert flat == views
    assert multi.shard([7], 1, 2) == [7]  # an empty share falls back to the whole list


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, _ = multi.dist_env()
    views = multi.shard(range(40), r, w)
    t = 1.0 + r  # rank 1 is the slow one
    out[rank] = (views, multi.max_over_ranks(t), multi.aggregate_rate(len(views), t, w))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    v0, m0, rate0 = out[0]
    v1, m1, rate1 = out[1]
    assert sorted(v0 + v1) == list(range(40)) and not set(v0) & set(v1)
    assert m0 == m1 == 2.0
    assert rate0 == rate1 == 20 * 2 / 2.0


def test_row_windows_cover_whole_tile_rows():
    for height in (1, 15, 16, 17, 180, 1080, 2160):
        for world in (1, 2, 3, 4, 8):
            wins = multi.row_windows(height, world)
            assert len(wins) == world
            rows = [r for r0, n in wins for r in range(r0, r0 + n)]
            assert rows == list(range(height))  # in order, disjoint, covering
            assert all(r0 % 16 == 0 for r0, n in wins if n)
            tiles = [(n + 15) // 16 for _, n in wins]  # tile rows per rank differ by one at most
            assert max(tiles) - min(tiles) <= 1


def _split_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, h = 37, 70

    def rows_of(row0, rows):  # a frame whose pixel (x, y) encodes y, x and the drawing rank
        y, x = np.meshgrid(np.arange(row0, row0 + rows), np.arange(w), indexing="ij")
        return np.stack([y % 256, x % 256, np.full_like(y, rank)], -1).astype(np.uint8)

    frame = multi.render_split(rows_of, w, h, rank, world)
    out[rank] = frame.tolist()
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_render_split_gathers_row_windows_over_two_ranks():
    import numpy as np

    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_split_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    wins = multi.row_windows(70, world)
    for r in range(world):
        f = np.array(out[r], np.uint8)
        assert f.shape == (70, 37, 3)
        assert np.array_equal(f[:, :, 0], (np.arange(70)[:, None] % 256).repeat(37, 1))
        for q, (r0, n) in enumerate(wins):  # each window drawn by its own rank
            assert np.all(f[r0:r0 + n, :, 2] == q)


# --- splat-sharded frames: the exchange's host logic --------------------------
# Toy splats stand in for the device: splat i covers pixel rows [y0, y1)
# (empty when y0 == y1) and its 48-byte record carries i. A rank's "window"
# encodes, per row, the sum and count of the splats received that cover it,
# and whether they arrived in scene order.

_RB = 48


def _toy_splats(n=500, height=70, seed=3):
    import numpy as np

    rng = np.random.default_rng(seed)
    y0 = rng.integers(-10, height + 5, n)
    y1 = y0 + rng.integers(0, 30, n)
    return np.clip(y0, 0, height), np.clip(y1, 0, height)


def _toy_rows(ids, y0, y1, row0, rows, width):
    import numpy as np

    out = np.zeros((rows, width, 3), np.uint8)
    for r in range(rows):
        cover = [i for i in ids if y0[i] <= row0 + r < y1[i]]
        out[r, :, 0] = sum(cover) % 256
        out[r, :, 1] = len(cover) % 256
        out[r, :, 2] = 1 if cover == sorted(cover) else 0
    return out


def _sharded_worker(rank, world, port, height, out):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    y0, y1 = _toy_splats(height=height)
    s0, s1 = multi.shard_range(len(y0), rank, world)
    width = 5

    def shard(bounds):
        runs, counts = [], []
        for k in range(len(bounds) - 1):
            ids = [i for i in range(s0, s1) if y0[i] < y1[i] and y0[i] < bounds[k + 1] and y1[i] > bounds[k]]
            rec = np.zeros((len(ids), _RB), np.uint8)
            rec[:, :8] = np.array(ids, np.int64).reshape(-1, 1).view(np.uint8)
            runs.append(rec)
            counts.append(len(ids))
        return torch.from_numpy(np.concatenate(runs).reshape(-1)), counts

    def draw(records, n, row0, rows):
        ids = records.numpy().reshape(n, _RB)[:, :8].copy().view(np.int64).reshape(-1).tolist()
        return torch.from_numpy(_toy_rows(ids, y0, y1, row0, rows, width))

    frame = multi.render_sharded(shard, draw, width, height, rank, world, _RB)
    out[rank] = frame.tolist()
    dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world,height", [(2, 70), (3, 70), (3, 40)])
def test_render_sharded_exchanges_records_over_gloo(world, height):
    import numpy as np

    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_sharded_worker, args=(world, _free_port(), height, out), nprocs=world,
                       start_method="spawn", join=True)
    y0, y1 = _toy_splats(height=height)
    want = _toy_rows(list(range(len(y0))), y0, y1, 0, height, 5)
    assert want[:, :, 1].max() > 0
    for r in range(world):
        assert np.array_equal(np.array(out[r], np.uint8), want), f"rank {r}"


def test_shard_range_covers_in_order():
    for n in (0, 1, 7, 1000):
        for world in (1, 2, 3, 8):
            parts = [multi.shard_range(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert max(b - a for a, b in parts) - min(b - a for a, b in parts) <= 1
