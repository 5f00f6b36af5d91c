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
