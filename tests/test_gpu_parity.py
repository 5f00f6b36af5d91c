"""Parity of the sm_100a backend with the oracle (the C++ restatement of the
reference's `cpu` and `cpu-naive` rasterizers), through the C ABI.

Gates:
* projection (x, y, conic, colour, opacity, depth, extents) bit-identical to
  the oracle's `project` for every splat, culling identical;
* sorted keys, values and tile ranges bit-identical to a CPU recomputation
  from the device's own projected x, y, extents and depths;
* images with SPLAT_OPT_EXACT_BLEND identical to the oracle `cpu` backend;
* default (FMA + hardware exp2) images >= 60 dB PSNR and max per-channel
  error <= 2/255 against the oracle `cpu` backend;
* the reference's own image tests (tests/render.rs) with the cuda backend.
"""

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis, View, to_radians
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu

MIN_PSNR = 60.0  # dB against the cpu backend
MAX_ERR = 2  # u8 levels against the cpu backend


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


_SCENES = {}


def scene(name):
    if name not in _SCENES:
        _SCENES[name] = {
            "lattice": lambda: __import__("splat_b200.synth", fromlist=["x"]).lattice_scene(),
            "clusters3": lambda: scenes.clusters(20_000, seed=7, sh_degree=3),
            "clusters1": lambda: scenes.clusters(8_000, seed=8, sh_degree=1),
            "clusters2": lambda: scenes.clusters(8_000, seed=9, sh_degree=2),
            "cube": scenes.cube,
            "galaxy": scenes.galaxy,
            "shballs": scenes.shballs,
        }[name]()
    return _SCENES[name]


def orbit_views(s, n=4):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    out = [cam.view()]
    for i in range(n - 1):
        cam.rotate(1.1, 0.0)
        cam.pitch = np.float32(0.5 * np.sin(i))
        cam.zoom(1.7 if i % 2 == 0 else 0.6)
        out.append(cam.view())
    return out


def pose_view(s, yaw, pitch, up):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, up)
    cam.rotate(yaw, np.float32(pitch) - cam.pitch)
    return cam.view()


def cuda_frame(r, view, w, h, bg=(0.0, 0.0, 0.0), exact=False, downsample=1):
    r.set_exact(exact)
    f = Frame()
    st = r.render(view, w, h, bg, f, downsample=downsample)
    return f.pixels.copy(), st


PROJ_CASES = [(name, size) for name in ["lattice", "clusters3", "clusters1", "clusters2", "shballs", "galaxy"]
              for size in [(320, 180), (37, 23), (1920, 1080)]]


@pytest.mark.parametrize("name,size", PROJ_CASES)
def test_projection_and_keys_bit_exact(oracle, name, size):
    s = scene(name)
    w, h = size
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    for view in orbit_views(s, 3):
        r.render(view, w, h, (0.1, 0.2, 0.3), Frame())
        d = r.debug_dump(w, h)
        ref, vis = oracle.project(s, view, w, h)
        assert np.array_equal(d["visible"], vis), f"{name}: culling differs"
        p = d["proj"][vis]
        o = ref[vis]
        # device: x, y, ext_x, ext_y, depth, conic a, b, c ; oracle: x, y, conic[3], color[3], op, depth, ext_x, ext_y
        pairs = [(0, 0), (1, 1), (2, 10), (3, 11), (4, 9), (5, 2), (6, 3), (7, 4)]
        for di, oi in pairs:
            assert np.array_equal(p[:, di].view(np.uint32), o[:, oi].view(np.uint32)), f"{name}: field {di} differs"
        assert np.array_equal(d["color"][vis].view(np.uint32), o[:, 5:8].view(np.uint32)), f"{name}: colour differs"
        # Keys / values / ranges against the CPU recomputation from the device's own projection.
        pr = d["proj"]
        keys, vals, ranges = oracle.bin_sort(pr[:, 0], pr[:, 1], pr[:, 2], pr[:, 3], pr[:, 4], d["visible"], w, h)
        assert np.array_equal(d["keys"], keys), f"{name}: keys differ"
        assert np.array_equal(d["values"], vals), f"{name}: values differ"
        assert np.array_equal(d["ranges"], ranges), f"{name}: ranges differ"
    r.close()


IMAGE_CASES = [("lattice", (320, 192)), ("clusters3", (640, 360)), ("shballs", (97, 53)), ("cube", (333, 77)),
               ("galaxy", (320, 180)), ("clusters1", (64, 48)), ("clusters2", (17, 9))]


@pytest.mark.parametrize("name,size", IMAGE_CASES)
def test_images_match_cpu_backend(oracle, name, size):
    s = scene(name)
    w, h = size
    r = CudaRenderer(s)
    cpu = oracle.CpuTiled(s)
    for view in orbit_views(s, 3):
        bg = (0.1, 0.2, 0.3)
        want, _ = cpu.render(view, w, h, bg)
        exact, st = cuda_frame(r, view, w, h, bg, exact=True)
        assert np.array_equal(exact, want), f"{name}: exact blend differs from cpu ({np.sum(exact != want)} channels)"
        fast, _ = cuda_frame(r, view, w, h, bg, exact=False)
        p = oracle.psnr(fast, want)
        err = int(np.max(np.abs(fast.astype(int) - want.astype(int))))
        assert p >= MIN_PSNR and err <= MAX_ERR, f"{name}: psnr {p} max err {err}"
    cpu.close()
    r.close()


def test_backends_agree_on_odd_sizes_and_poses(oracle):
    """tests/render.rs:45-67 with the cuda backend against cpu-naive (45 dB, the
    reference's own threshold) and against cpu (60 dB)."""
    for name in ["cube", "galaxy"]:
        s = scene(name)
        r = CudaRenderer(s)
        cpu = oracle.CpuTiled(s)
        for (w, h) in [(1, 1), (17, 9), (16, 16), (33, 31), (64, 48), (333, 77)]:
            for yaw, pitch, up in [(0.37, 0.26, UpAxis.NEG_Y), (1.3, -0.5, UpAxis.NEG_Y), (4.0, 0.9, UpAxis.POS_Y),
                                   (2.0, 0.1, UpAxis.POS_Z), (5.5, 0.3, UpAxis.NEG_Z)]:
                v = pose_view(s, yaw, pitch, up)
                bg = (0.1, 0.2, 0.3)
                a, _ = cuda_frame(r, v, w, h, bg)
                b, _ = oracle.render_naive(s, v, w, h, bg)
                c, _ = cpu.render(v, w, h, bg)
                assert oracle.psnr(a, b) >= 45.0, f"{name} {w}x{h} {yaw} {pitch} {up}"
                assert oracle.psnr(a, c) >= MIN_PSNR, f"{name} {w}x{h} {yaw} {pitch} {up}"
        cpu.close()
        r.close()


def test_equal_depth_ties_match_reference(oracle):
    """src/render/mod.rs:366-392: the cube lattice seen down an axis has many
    bit-identical depths; ties blend in scene-index order."""
    s = scene("cube")
    c, rad = s.bounds()
    cam = OrbitCamera.new(c, rad, UpAxis.NEG_Y)
    views = [cam.view()]
    cam.pitch = np.float32(0.0)
    cam.yaw = np.float32(0.0)
    views.append(cam.view())
    r = CudaRenderer(s)
    cpu = oracle.CpuTiled(s)
    for v in views:
        for (w, h) in [(37, 23), (64, 64), (160, 90)]:
            want, _ = cpu.render(v, w, h)
            got, _ = cuda_frame(r, v, w, h, exact=True)
            assert np.array_equal(got, want)
            again, _ = cuda_frame(r, v, w, h, exact=True)
            assert np.array_equal(again, got), "nondeterministic"
            naive, _ = oracle.render_naive(s, v, w, h)
            fast, _ = cuda_frame(r, v, w, h)
            assert oracle.psnr(naive, fast) >= 45.0
    r.close()
    cpu.close()


@pytest.mark.parametrize("factor", [0, 1, 2, 3, 4, 8, 16])
def test_fused_downsample_matches_term_downsample(oracle, factor):
    s = scene("clusters3")
    v = orbit_views(s, 2)[1]
    r = CudaRenderer(s)
    for (w, h) in [(320, 192), (333, 77), (37, 23)]:
        full, _ = cuda_frame(r, v, w, h, (0.2, 0.4, 0.6), exact=True)
        small, _ = cuda_frame(r, v, w, h, (0.2, 0.4, 0.6), exact=True, downsample=factor)
        want = oracle.downsample(full, factor)
        assert small.shape == want.shape
        assert np.array_equal(small, want), f"{w}x{h} f={factor}"
    r.close()


def test_pair_buffers_grow_and_rerender(oracle):
    s = scene("clusters3")
    v = orbit_views(s, 1)[0]
    big = CudaRenderer(s)
    ref, st = cuda_frame(big, v, 640, 360, exact=True)
    small = CudaRenderer(s)
    small.set_option(N.SPLAT_OPT_PAIR_CAPACITY, 64)
    got, st2 = cuda_frame(small, v, 640, 360, exact=True)
    assert np.array_equal(got, ref)
    assert st2.overlaps == st.overlaps
    assert small.get_option(N.SPLAT_OPT_PAIR_CAPACITY) >= st.overlaps
    big.close()
    small.close()


def test_stats_match_cpu_backend(oracle):
    s = scene("clusters3")
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    cpu = oracle.CpuTiled(s)
    for v in orbit_views(s, 3):
        _, st = cuda_frame(r, v, 320, 180)
        _, cst = cpu.render(v, 320, 180)
        assert st.visible == cst["visible"] and st.overlaps == cst["overlaps"]
        assert st.project_ms >= 0 and st.sort_ms >= 0 and st.raster_ms > 0 and st.total_ms > 0
    r.close()
    cpu.close()


# --- tests/render.rs image semantics, cuda backend ------------------------------------
RED = (1.0, 0.0, 0.0)
BLUE = (0.0, 0.0, 1.0)


def render_scene(items, view, w, h, bg):
    r = CudaRenderer(scenes.splats(items) if items else scenes.empty())
    f = Frame()
    st = r.render(view, w, h, bg, f)
    assert (f.width, f.height) == (w, h)
    r.close()
    return f, st


def test_single_red_splat_center_red_corners_background():
    v = View.looking_along_z((0, 0, 0))
    for (w, h) in [(64, 64), (65, 33), (200, 100)]:
        f, _ = render_scene([((0, 0, 5), 0.5, 1.0, RED)], v, w, h, (0, 0, 0))
        c = f.get(w // 2, h // 2)
        assert c[0] > 200 and c[1] < 10 and c[2] < 10
        for (x, y) in [(0, 0), (w - 1, 0), (0, h - 1), (w - 1, h - 1)]:
            assert f.get(x, y) == [0, 0, 0]


def test_background_color_shows_through():
    f, _ = render_scene([((0, 0, 5), 0.5, 1.0, RED)], View.looking_along_z((0, 0, 0)), 64, 64, (0, 1, 0))
    assert f.get(0, 0) == [0, 255, 0]


def test_splat_behind_camera_renders_nothing():
    f, st = render_scene([((0, 0, -5), 0.5, 1.0, RED)], View.looking_along_z((0, 0, 0)), 40, 30, (0.5, 0.5, 0.5))
    assert st.visible == 0
    assert np.all(f.pixels == 128)


def test_off_screen_and_transparent_splats_give_pure_background():
    f, _ = render_scene([((500, 0, 5), 0.5, 1.0, RED), ((0, 0, 5), 0.5, 0.0, RED)],
                        View.looking_along_z((0, 0, 0)), 50, 50, (0.2, 0.4, 0.6))
    assert np.all(f.pixels == f.pixels[0, 0])


def test_empty_scene_is_background():
    f, st = render_scene([], View.looking_along_z((0, 0, 0)), 20, 10, (1, 1, 1))
    assert np.all(f.pixels == 255) and st.visible == 0


def test_near_opaque_blue_hides_far_red_regardless_of_insertion_order():
    blue = ((0, 0, 4), 0.5, 1.0, BLUE)
    red = ((0, 0, 8), 1.0, 1.0, RED)
    for order in ([blue, red], [red, blue]):
        f, _ = render_scene(order, View.looking_along_z((0, 0, 0)), 64, 64, (0, 0, 0))
        c = f.get(32, 32)
        assert c[2] > 200 and c[0] < 10


def test_translucent_front_blends_with_back():
    f, _ = render_scene([((0, 0, 4), 0.5, 0.5, BLUE), ((0, 0, 8), 2.0, 1.0, RED)], View.looking_along_z((0, 0, 0)),
                        64, 64, (0, 0, 0))
    c = f.get(32, 32)
    assert c[0] > 40 and c[2] > 40


def test_splat_moves_with_camera_translation():
    f, _ = render_scene([((1, 0, 5), 0.2, 1.0, RED)], View.looking_along_z((0, 0, 0)), 100, 100, (0, 0, 0))
    red = f.pixels[:, :, 0] > 100
    assert red[:, 50:].sum() > 0 and red[:, :50].sum() == 0


def test_repeated_renders_are_deterministic_and_resize_safe():
    s = scene("cube")
    c, rad = s.bounds()
    v = OrbitCamera.new(c, rad, UpAxis.NEG_Y).view()
    r = CudaRenderer(s)
    f = Frame()
    r.render(v, 48, 32, (0, 0, 0), f)
    first = f.pixels.copy()
    r.render(v, 7, 5, (0, 0, 0), f)
    assert (f.width, f.height, f.pixels.shape) == (7, 5, (5, 7, 3))
    r.render(v, 48, 32, (0, 0, 0), f)
    assert np.array_equal(f.pixels, first)
    r.close()


def test_zero_size_render_and_pixel_limit():
    """src/render/mod.rs:349-364 and 398-409."""
    s = scene("cube")
    r = CudaRenderer(s)
    v = orbit_views(s, 1)[0]
    for (w, h) in [(0, 0), (64, 0), (0, 64)]:
        f = Frame()
        st = r.render(v, w, h, (0, 0, 0), f)
        assert f.pixels.size == 0 and st.visible == 0
    with pytest.raises(ValueError, match="pixel limit"):
        r.render(v, 65536, 65537, (0, 0, 0), Frame())
    # The C ABI itself rejects oversized frames with INVALID_ARG.
    import ctypes

    buf = np.zeros(16, np.uint8)
    bg = np.zeros(3, np.float32)
    from splat_b200.render import _view_desc

    rc = N.lib().splat_cuda_render(r._h, ctypes.byref(_view_desc(v)), 16385, 1,
                                   bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), 1, buf.ctypes.data, buf.nbytes,
                                   None)
    assert rc == N.SPLAT_ERR_INVALID_ARG
    assert "pixel limit" in N.lib().splat_cuda_last_error(r._h).decode()
    r.close()


def test_max_frame_dims_allowed():
    s = scenes.splats([((0, 0, 5), 0.5, 1.0, RED)])
    r = CudaRenderer(s)
    f = Frame()
    r.render(View.looking_along_z((0, 0, 0)), 16384, 1, (0, 0, 0), f)
    assert f.pixels.shape == (1, 16384, 3)
    r.close()


def test_device_path_matches_host_path():
    import torch

    s = scene("clusters3")
    v = orbit_views(s, 2)[1]
    r = CudaRenderer(s)
    host, _ = cuda_frame(r, v, 320, 180, (0.1, 0.1, 0.1))
    out = torch.zeros(320 * 180 * 3, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    r.render_device(v, 320, 180, (0.1, 0.1, 0.1), out.data_ptr(), out.numel())
    st, regrown = r.finish()
    assert not regrown
    assert np.array_equal(out.cpu().numpy().reshape(180, 320, 3), host)
    pinned = torch.zeros(320 * 180 * 3, dtype=torch.uint8).pin_memory()
    r.render_into(v, 320, 180, (0.1, 0.1, 0.1), pinned.data_ptr(), pinned.numel())
    assert np.array_equal(pinned.numpy().reshape(180, 320, 3), host)
    r.close()


@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("cfg", [(16, 16, 512), (8, 8, 256), (32, 16, 256)])
def test_row_windows_match_the_whole_frame(exact, cfg):
    """splat_cuda_render_rows: any window of rows (tile-aligned or not, one
    row, the whole frame) equals those rows of the whole frame bit for bit,
    and windows that split the frame (multi.row_windows, as ranks would draw
    them) stitch back into it."""
    from splat_b200 import multi

    s = scene("clusters3")
    w, h = 333, 191
    r = CudaRenderer(s)
    r.set_blend_config(*cfg)
    for v in orbit_views(s, 2):
        full, _ = cuda_frame(r, v, w, h, (0.1, 0.2, 0.3), exact=exact)
        for row0, rows in [(0, h), (16, 32), (5, 50), (190, 1), (47, 144)]:
            got = r.render_rows(v, w, h, (0.1, 0.2, 0.3), row0, rows)
            assert np.array_equal(got, full[row0:row0 + rows]), (row0, rows)
        for world in (2, 3, 4):
            parts = [r.render_rows(v, w, h, (0.1, 0.2, 0.3), r0, n) for r0, n in multi.row_windows(h, world) if n]
            assert np.array_equal(np.concatenate(parts), full)
        # a window into mapped pinned memory (written by the kernels directly)
        import torch

        pinned = torch.full((64, w, 3), 7, dtype=torch.uint8).pin_memory().numpy()
        r.render_rows(v, w, h, (0.1, 0.2, 0.3), 32, 64, out=pinned)
        assert np.array_equal(pinned, full[32:96])
    with pytest.raises(N.SplatError, match="exceed the frame height"):
        r.render_rows(orbit_views(s, 1)[0], w, h, (0, 0, 0), 150, 50)
    r.close()


@pytest.mark.parametrize("size,f,cfg", [((1920, 1080), 1, (16, 16, 512)), ((1920, 1080), 1, (32, 16, 256)),
                                        ((1920, 1080), 1, (8, 8, 256)), ((333, 191), 1, (16, 16, 512)),
                                        ((320, 192), 2, (16, 16, 512)), ((333, 191), 3, (16, 16, 512))])
def test_frame_written_into_mapped_pinned_memory(size, f, cfg):
    """Pinned host output is written by the kernels through its device
    mapping (4-byte words of tile rows where the rows are aligned, bytes
    elsewhere): the frame equals the one copied out of device memory and the
    one staged for pageable memory, at aligned and ragged widths and with the
    fused and unfused downsample."""
    import torch

    s = scene("clusters3")
    w, h = size
    ow, oh = w // f, h // f
    r = CudaRenderer(s)
    r.set_blend_config(*cfg)
    for v in orbit_views(s, 3)[1:]:
        host, _ = cuda_frame(r, v, w, h, (0.1, 0.2, 0.3), downsample=f)
        dev = torch.zeros(ow * oh * 3, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        r.render_device(v, w, h, (0.1, 0.2, 0.3), dev.data_ptr(), dev.numel(), downsample=f)
        _, regrown = r.finish()
        assert not regrown
        pinned = torch.full((ow * oh * 3,), 7, dtype=torch.uint8).pin_memory()
        for _ in range(2):
            r.render_into(v, w, h, (0.1, 0.2, 0.3), pinned.data_ptr(), pinned.numel(), downsample=f)
            assert np.array_equal(pinned.numpy().reshape(oh, ow, 3), host)
        assert np.array_equal(dev.cpu().numpy().reshape(oh, ow, 3), host)
    r.close()


@pytest.mark.parametrize("mode", ["truecolor", "ansi256"])
@pytest.mark.parametrize("size,f", [((320, 192), 2), ((333, 191), 3), ((161, 95), 1)])
def test_terminal_cells_match_widget(oracle, mode, size, f):
    """splat_cuda_render_cells: the HalfBlockImage cells (src/term.rs:109-130)
    of the term::downsample'd frame, truecolor and xterm-256."""
    from oracle import term_oracle as T
    from splat_b200 import _native as N

    s = scenes.clusters(20_000, seed=11, sh_degree=2)
    r = CudaRenderer(s)
    v = orbit_views(s, 2)[1]
    w, h = size
    frame = Frame()
    r.render(v, w, h, (0.05, 0.1, 0.2), frame, downsample=f)
    m = N.SPLAT_CELLS_TRUECOLOR if mode == "truecolor" else N.SPLAT_CELLS_ANSI256
    got = r.render_cells(v, w, h, (0.05, 0.1, 0.2), downsample=f, mode=m)
    want = T.cells(frame.pixels, mode)
    assert got.shape == want.shape and np.array_equal(got, want)
    r.close()


def test_c_driver_matches_python_path(tmp_path):
    """The C host renders the same frame and cells as the ctypes path."""
    import subprocess

    from splat_b200 import View
    from splat_b200.scene import Scene
    from tests import c_driver

    exe = c_driver.build(str(tmp_path))
    fr, ce = str(tmp_path / "frame.rgb"), str(tmp_path / "cells.bin")
    out = subprocess.run([exe, fr, ce], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    side = 8
    s = Scene()
    idx = np.arange(side ** 3)
    x, y, z = idx % side, (idx // side) % side, idx // (side * side)
    lin = lambda a: (np.float32(-1.0) + np.float32(2.0) * a.astype(np.float32) / np.float32(side - 1))  # noqa: E731
    s.positions = np.stack([lin(x), lin(y), lin(z)], 1).astype(np.float32)
    s.scales = np.full((side ** 3, 3), 0.05, np.float32)
    s.rotations = np.tile(np.array([0, 0, 0, 1], np.float32), (side ** 3, 1))
    s.opacities = np.full(side ** 3, 0.9, np.float32)
    s.colors = (np.stack([x, y, z], 1).astype(np.float32) / np.float32(side - 1)).astype(np.float32)
    s.finalize()
    r = CudaRenderer(s)
    v = View.from_array(np.array([0, 0, -4, 1, 0, 0, 0, 1, 0, 0, 0, 1, np.float32(50.0) * np.float32(3.14159265)
                                  / np.float32(180.0), 0.05], np.float32))
    f = Frame()
    r.render(v, 160, 96, (0.1, 0.1, 0.1), f)
    got = np.fromfile(fr, np.uint8).reshape(96, 160, 3)
    assert np.array_equal(got, f.pixels)
    cells = r.render_cells(v, 160, 96, (0.1, 0.1, 0.1), mode=N.SPLAT_CELLS_ANSI256)
    assert np.array_equal(np.fromfile(ce, np.uint8).reshape(cells.shape), cells)
    r.close()
