"""One frame from splats sharded over devices (splat_cuda_shard_records /
splat_cuda_render_records), with the devices emulated in one process on
one GPU: each shard's renderer selects its records for every row window,
the records of window k are concatenated in shard order (the all-to-all),
and window k is drawn from them. The assembled frame must equal the
one-device frame of the whole scene bit for bit, in the default and the
exact blend, for FP32 and FP16 storage, any blend shape, uneven and empty
windows, and windows drawn past the pair limit; the pair and visible counts
must add up to the whole frame's.

The last test runs two processes on the one GPU, exchanging through gloo
(host memory): no kernel of one process waits for the other's."""

import os
import socket

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200 import multi, synth
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu

RB = N.SPLAT_RECORD_BYTES


def _view(scene, yaw=0.4, zoom=1.0):
    c, r = scene.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.rotate(yaw, 0.0)
    if zoom != 1.0:
        cam.zoom(zoom)
    return cam.view()


def _emulated(scene, view, w, h, world, bounds=None, bg=(0.05, 0.1, 0.2), exact=False, blend=None,
              pair_limit=None):
    """The sharded frame with `world` shards on one GPU; returns (frame,
    per-window stats, summed shard visible counts)."""
    import torch

    if bounds is None:
        wins = multi.row_windows(h, world)
        bounds = [r0 for r0, _ in wins] + [h]
    n = len(scene)
    shards = [CudaRenderer(scene.shard(*multi.shard_range(n, r, world))) for r in range(world)]
    try:
        sends = [s.shard_records(view, w, h, bounds) for s in shards]
        frame = np.zeros((h, w, 3), np.uint8)
        stats = []
        for k in range(len(bounds) - 1):
            runs = []
            for send, counts, _ in sends:
                off = sum(counts[:k]) * RB
                runs.append(send[off:off + counts[k] * RB])
            recs = torch.cat(runs) if runs else torch.empty(0, dtype=torch.uint8, device="cuda")
            row0, rows = bounds[k], bounds[k + 1] - bounds[k]
            r = shards[k % world]
            r.set_exact(exact)
            if blend:
                r.set_blend_config(*blend)
            if pair_limit:
                r.set_option(N.SPLAT_OPT_PAIR_LIMIT, pair_limit)
            if rows:
                frame[row0:row0 + rows], st = r.render_records(view, w, h, bg, recs, row0, rows, stats=True)
                assert st.visible == recs.numel() // RB
                stats.append(st)
        return frame, stats, sum(v for _, _, v in sends)
    finally:
        for s in shards:
            s.close()


def _whole(scene, view, w, h, bg=(0.05, 0.1, 0.2), exact=False):
    r = CudaRenderer(scene)
    try:
        r.set_exact(exact)
        frame = Frame()
        st = r.render(view, w, h, bg, frame)
        return frame.pixels.copy(), st
    finally:
        r.close()


@pytest.fixture(scope="module")
def clusters():
    return scenes.clusters(20_000, seed=7, sh_degree=3)


@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_sharded_frame_equals_whole_frame(clusters, world):
    view = _view(clusters)
    want, st = _whole(clusters, view, 640, 360)
    got, wst, vis = _emulated(clusters, view, 640, 360, world)
    assert np.array_equal(got, want)
    assert vis == st.visible
    assert sum(s.overlaps for s in wst) == st.overlaps  # tile-aligned windows: the same pairs


def test_sharded_frame_exact_blend(clusters):
    view = _view(clusters, yaw=2.0)
    want, _ = _whole(clusters, view, 480, 272, exact=True)
    got, _, _ = _emulated(clusters, view, 480, 272, 3, exact=True)
    assert np.array_equal(got, want)


def test_sharded_frame_fp16(clusters):
    half = clusters.to_fp16()
    view = _view(clusters, yaw=1.1)
    want, _ = _whole(half, view, 512, 288)
    got, _, _ = _emulated(half, view, 512, 288, 2)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("blend", [(8, 8, 256), (32, 16, 512), (16, 16, 128)])
def test_sharded_frame_any_blend_shape(clusters, blend):
    view = _view(clusters, yaw=-0.7)
    want, _ = _whole(clusters, view, 400, 300)
    got, _, _ = _emulated(clusters, view, 400, 300, 2, blend=blend)
    assert np.array_equal(got, want)


def test_sharded_frame_uneven_and_empty_windows(clusters):
    view = _view(clusters, yaw=0.9)
    want, _ = _whole(clusters, view, 320, 200)
    # windows not aligned to tiles, an empty one, one of a single row
    got, _, _ = _emulated(clusters, view, 320, 200, 3, bounds=[0, 37, 37, 38, 131, 200])
    assert np.array_equal(got, want)
    # more ranks than tile rows: row_windows gives some ranks no rows
    want, _ = _whole(clusters, view, 320, 40)
    got, _, _ = _emulated(clusters, view, 320, 40, 4)
    assert np.array_equal(got, want)


def test_sharded_windows_past_the_pair_limit(clusters):
    view = _view(clusters, yaw=0.2, zoom=0.6)
    want, st = _whole(clusters, view, 640, 360)
    got, wst, _ = _emulated(clusters, view, 640, 360, 2, pair_limit=max(1024, st.overlaps // 8))
    assert np.array_equal(got, want)
    assert sum(s.overlaps for s in wst) == st.overlaps


def test_send_capacity_is_reported(clusters):
    import ctypes

    import torch

    r = CudaRenderer(clusters.shard(0, 5000))
    try:
        view = _view(clusters)
        bounds = np.array([0, 100, 360], np.uint32)
        counts = np.zeros(2, np.uint64)
        vis = ctypes.c_uint64(0)
        buf = torch.empty(64 * RB, dtype=torch.uint8, device="cuda")
        from splat_b200.render import _view_desc

        rc = N.lib().splat_cuda_shard_records(r._h, ctypes.byref(_view_desc(view)), 640, 360, 2,
                                              bounds.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                              buf.data_ptr(), 64, counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                              ctypes.byref(vis))
        assert rc == N.SPLAT_ERR_CAPACITY and counts.sum() > 64 and vis.value > 0
        # the wrapper sizes its buffer from the counts and calls again
        send, c2, v2 = r.shard_records(view, 640, 360, bounds, send=buf)
        assert c2 == [int(c) for c in counts] and v2 == vis.value and send.numel() == counts.sum() * RB
        # bad bounds are rejected before any work
        bad = np.array([0, 200, 100], np.uint32)
        with pytest.raises(N.SplatError) as e:
            r.shard_records(view, 640, 360, bad)
        assert e.value.code == N.SPLAT_ERR_INVALID_ARG
    finally:
        r.close()


def test_sharded_headline_scene():
    """The 1.2M-splat SH3 scene at 1920x1080 over 4 shards."""
    scene = synth.cluster_scene(1_200_000, seed=0x5EED0001, sh_degree=3)
    cam = synth.orbit_camera(scene)
    home, _, timed = synth.orbit_views(cam, 40, 5)
    for view in (home, timed[7]):
        want, st = _whole(scene, view, 1920, 1080, bg=(0.0, 0.0, 0.0))
        got, wst, vis = _emulated(scene, view, 1920, 1080, 4, bg=(0.0, 0.0, 0.0))
        assert np.array_equal(got, want)
        assert vis == st.visible and sum(s.overlaps for s in wst) == st.overlaps


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    scene = scenes.clusters(20_000, seed=7, sh_degree=3)
    view = _view(scene, yaw=1.7)
    r = CudaRenderer(scene.shard(*multi.shard_range(len(scene), rank, world)))
    frame, vis, pairs = multi.render_sharded_frame(r, view, 640, 360, (0.0, 0.0, 0.0), rank, world)
    r.close()
    out[rank] = (frame.tobytes(), vis, pairs)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_processes_over_gloo():
    import torch.multiprocessing as mp

    world = 2
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_gloo_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    scene = scenes.clusters(20_000, seed=7, sh_degree=3)
    want, st = _whole(scene, _view(scene, yaw=1.7), 640, 360, bg=(0.0, 0.0, 0.0))
    for r in range(world):
        assert out[r][0] == want.tobytes(), f"rank {r}"
    assert sum(out[r][1] for r in range(world)) == st.visible
    assert sum(out[r][2] for r in range(world)) == st.overlaps
