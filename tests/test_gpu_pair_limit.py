"""Frames that need more (splat, tile) pairs than the pair buffers may hold.

The reference's gpu backend saturates its pair count and renders only the
front-most pairs past its capacity limit (src/render/gpu.rs:1253-1289,
`gpu_degrades_gracefully_past_pair_limits`; its test lowers the limit with
`max_cap = 1 << 18`). Here such a frame is drawn in windows of whole tiles
whose pairs fit, each window with the whole frame's projection, so the frame
is complete: identical to the one-pass frame and to the oracle `cpu`
backend, with `overlaps` counting every pair.
"""

import ctypes

import numpy as np
import pytest

from splat_b200 import Frame, View
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from splat_b200.scene import Scene
from tests import scenes

pytestmark = pytest.mark.gpu

f32 = np.float32


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def plane_view():
    """src/render/gpu.rs:1162-1171 with dist 0."""
    return View(np.zeros(3, f32), np.array([1, 0, 0], f32), np.array([0, 1, 0], f32), np.array([0, 0, 1], f32),
                f32(1.0), f32(0.01))


def screen_filling(n):
    """src/render/gpu.rs:1256-1263: n isotropic splats of scale 50 on the
    optical axis at depth 1 + i * 1e-4, opacity 0.9, the nearest red, the
    others green."""
    s = Scene()
    i = np.arange(n, dtype=f32)
    s.positions = np.stack([np.zeros(n, f32), np.zeros(n, f32), f32(1.0) + i * f32(1e-4)], 1)
    s.scales = np.full((n, 3), 50.0, f32)
    s.rotations = np.tile(np.array([0, 0, 0, 1], f32), (n, 1))
    s.opacities = np.full(n, 0.9, f32)
    s.colors = np.tile(np.array([0, 1, 0], f32), (n, 1))
    s.colors[0] = (1, 0, 0)
    return s.finalize()


def test_frame_past_the_pair_limit_is_complete(oracle):
    """The reference's scenario at 256x256 with its lowered limit (1 << 18
    pairs): 70k splats cover all 256 tiles (17.9M pairs), a tile row holds
    1.1M pairs, so windows shrink to a few tiles of a row."""
    n, w, h = 70_000, 256, 256
    s = screen_filling(n)
    v = plane_view()
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    r.set_option(N.SPLAT_OPT_PAIR_LIMIT, 1 << 18)
    assert r.get_option(N.SPLAT_OPT_PAIR_LIMIT) == 1 << 18
    cpu = oracle.CpuTiled(s)
    try:
        want, cst = cpu.render(v, w, h, (0.0, 0.0, 0.0))
        f = Frame()
        r.set_exact(True)
        st = r.render(v, w, h, (0.0, 0.0, 0.0), f)
        assert st.visible == n
        assert st.overlaps == cst["overlaps"] == n * (w // 16) * (h // 16)
        assert r.get_option(N.SPLAT_OPT_PAIR_CAPACITY) <= 1 << 18
        assert np.array_equal(f.pixels, want), f"exact blend differs in {np.sum(f.pixels != want)} channels"
        r.set_exact(False)
        fast = Frame()
        r.render(v, w, h, (0.0, 0.0, 0.0), fast)
        assert oracle.psnr(fast.pixels, want) >= 60.0
        assert int(np.max(np.abs(fast.pixels.astype(int) - want.astype(int)))) <= 2
        c = fast.pixels[h // 2, w // 2]
        assert c[0] > 200 and c[1] < 60 and c[2] == 0, f"center pixel {c}"
        again = Frame()
        r.render(v, w, h, (0.0, 0.0, 0.0), again)
        assert np.array_equal(again.pixels, fast.pixels), "repeated renders differ"
    finally:
        cpu.close()
        r.close()


def test_reference_pair_limit_scenario_full_size():
    """src/render/gpu.rs:1253-1289 at its own size: 70k screen-filling
    splats at 2048x2048. With 16x16 tiles that is 70k x 16384 = 1.15e9
    pairs, above the 2^30 - 1 pair limit: the frame is drawn in windows and
    every pair is counted (the reference saturates at 2^32 - 1 and keeps the
    front-most pairs). The centre pixel check is the reference's."""
    n, w, h = 70_000, 2048, 2048
    s = screen_filling(n)
    v = plane_view()
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    try:
        f = Frame()
        st = r.render(v, w, h, (0.0, 0.0, 0.0), f)
        assert st.visible == n
        assert st.overlaps == n * (w // 16) * (h // 16) > (1 << 30) - 1
        assert r.get_option(N.SPLAT_OPT_PAIR_CAPACITY) <= (1 << 30) - 1
        c = f.pixels[h // 2, w // 2]
        assert c[0] > 200 and c[1] < 60 and c[2] == 0, f"center pixel {c}"
        again = Frame()
        r.render(v, w, h, (0.0, 0.0, 0.0), again)
        assert np.array_equal(again.pixels, f.pixels), "repeated renders differ"
    finally:
        r.close()


@pytest.fixture(scope="module")
def clusters():
    return scenes.clusters(20_000, seed=7, sh_degree=3)


def _view(s):
    from splat_b200 import OrbitCamera, UpAxis

    c, rad = s.bounds()
    cam = OrbitCamera.new(c, rad, UpAxis.NEG_Y)
    cam.zoom(0.6)
    return cam.view()


def test_windows_on_every_output_path(clusters):
    """With the limit at a fifth of the frame's pairs, every entry point
    draws the frame in windows and gives what it gives in one pass: host
    frames (pageable and mapped pinned), device frames (render_device +
    finish), row windows, fused (f = 2) and unfused (f = 3) downsampling,
    terminal cells."""
    import torch

    s = clusters
    v = _view(s)
    w, h = 640, 360
    bg = (0.1, 0.2, 0.3)
    one = CudaRenderer(s)
    win = CudaRenderer(s)
    try:
        base = Frame()
        st = one.render(v, w, h, bg, base)
        limit = max(1024, st.overlaps // 5)
        win.set_option(N.SPLAT_OPT_PAIR_LIMIT, limit)
        got = Frame()
        st2 = win.render(v, w, h, bg, got)
        assert st2.overlaps == st.overlaps and st2.visible == st.visible
        assert np.array_equal(got.pixels, base.pixels)
        # mapped pinned host memory (the blend writes the frame through the device mapping)
        pinned = torch.empty(w * h * 3, dtype=torch.uint8).pin_memory()
        win.render_into(v, w, h, bg, pinned.data_ptr(), pinned.numel())
        assert np.array_equal(pinned.numpy().reshape(h, w, 3), base.pixels)
        # device frame: render_device + finish redraws the last frame in windows
        dev = torch.zeros(w * h * 3, dtype=torch.uint8, device="cuda")
        win.render_device(v, w, h, bg, dev.data_ptr(), dev.numel())
        dst, regrown = win.finish()
        assert not regrown and dst.overlaps == st.overlaps
        assert np.array_equal(dev.cpu().numpy().reshape(h, w, 3), base.pixels)
        # a window of rows (not aligned to tiles)
        rows = win.render_rows(v, w, h, bg, 37, 250)
        assert np.array_equal(rows, base.pixels[37:287])
        for f in (2, 3):
            a, b = Frame(), Frame()
            one.render(v, w, h, bg, a, downsample=f)
            win.render(v, w, h, bg, b, downsample=f)
            assert np.array_equal(a.pixels, b.pixels), f"downsample {f}"
        ca = one.render_cells(v, w, h, bg, downsample=2, mode=N.SPLAT_CELLS_ANSI256)
        cb = win.render_cells(v, w, h, bg, downsample=2, mode=N.SPLAT_CELLS_ANSI256)
        assert np.array_equal(ca, cb)
    finally:
        one.close()
        win.close()


def test_a_tile_beyond_the_limit_is_an_error():
    """A single tile with more pairs than the pair buffers may hold cannot be
    split further: SPLAT_ERR_CAPACITY, and the handle renders afterwards."""
    s = screen_filling(3000)
    v = plane_view()
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    try:
        r.set_option(N.SPLAT_OPT_PAIR_LIMIT, 2048)
        with pytest.raises(N.SplatError) as e:
            r.render(v, 64, 64, (0.0, 0.0, 0.0), Frame())
        assert e.value.code == N.SPLAT_ERR_CAPACITY
        r.set_option(N.SPLAT_OPT_PAIR_LIMIT, (1 << 30) - 1)
        st = r.render(v, 64, 64, (0.0, 0.0, 0.0), Frame())
        assert st.overlaps == 3000 * 16
    finally:
        r.close()


def test_pair_limit_option_bounds():
    r = CudaRenderer(scenes.clusters(1000, seed=1, sh_degree=0))
    try:
        for bad in (0, 1023, 1 << 30):
            assert N.lib().splat_cuda_set_option(r._h, N.SPLAT_OPT_PAIR_LIMIT, bad) == N.SPLAT_ERR_INVALID_ARG
        r.set_option(N.SPLAT_OPT_PAIR_LIMIT, 4096)
        assert N.lib().splat_cuda_set_option(r._h, N.SPLAT_OPT_PAIR_CAPACITY, 8192) == N.SPLAT_ERR_INVALID_ARG
        r.set_option(N.SPLAT_OPT_PAIR_CAPACITY, 4096)
        v = ctypes.c_uint64(0)
        assert N.lib().splat_cuda_get_option(r._h, N.SPLAT_OPT_PAIR_CAPACITY, ctypes.byref(v)) == N.SPLAT_OK
        assert v.value == 4096
    finally:
        r.close()
