"""Tile shapes, blend thread counts and the batched (CUDA graph) path.

Gates:
* every blend configuration (8x8, 16x16, 32x16 tiles x 128, 256, 512
  threads) draws exact-blend images identical to the oracle `cpu` backend,
  default images >= 60 dB / <= 2/255 against it, and keys/ranges bit-exact
  against the CPU recomputation with that tile shape;
* a batch of views of uneven resolution over scenes of different SH degree
  and storage precision draws, for every view, exactly the image the single
  view path draws, with the same visible and pair counts; replays of the
  recorded graph repeat it; every configuration of the batch draws the same
  images; the tuner reports every configuration and keeps the fastest.
"""

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200.batch import BatchRenderer, BatchView
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _view(s, yaw, pitch, zoom):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.rotate(yaw, pitch)
    cam.zoom(zoom)
    return cam.view()


@pytest.mark.parametrize("cfg", N.BLEND_CONFIGS)
def test_blend_configs_match_cpu_backend(oracle, cfg):
    s = scenes.clusters(20_000, seed=41, sh_degree=3)
    r = CudaRenderer(s)
    r.set_blend_config(*cfg)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    cpu = oracle.CpuTiled(s)
    for i, (w, h) in enumerate([(333, 190), (64, 48), (17, 9)]):
        v = _view(s, 0.7 * i, 0.2, 0.6 + 0.4 * i)
        want, _ = cpu.render(v, w, h, (0.1, 0.2, 0.3))
        r.set_exact(True)
        f = Frame()
        st = r.render(v, w, h, (0.1, 0.2, 0.3), f)
        assert np.array_equal(f.pixels, want), f"{cfg} {w}x{h}: {np.sum(f.pixels != want)} channels differ"
        d = r.debug_dump(w, h)
        pr = d["proj"]
        keys, vals, ranges = oracle.bin_sort(pr[:, 0], pr[:, 1], pr[:, 2], pr[:, 3], pr[:, 4], d["visible"], w, h,
                                             tile=cfg[:2])
        assert np.array_equal(d["keys"], keys) and np.array_equal(d["values"], vals), f"{cfg}: keys differ"
        assert np.array_equal(d["ranges"], ranges), f"{cfg}: ranges differ"
        assert st.overlaps == len(keys)
        r.set_exact(False)
        r.render(v, w, h, (0.1, 0.2, 0.3), f)
        p = oracle.psnr(f.pixels, want)
        err = int(np.max(np.abs(f.pixels.astype(int) - want.astype(int))))
        assert p >= 60.0 and err <= 2, (cfg, p, err)
    cpu.close()
    r.close()


@pytest.mark.parametrize("cfg", [(8, 8, 256), (32, 16, 128)])
@pytest.mark.parametrize("f", [2, 4, 3])
def test_blend_configs_downsample(oracle, cfg, f):
    s = scenes.clusters(8_000, seed=43, sh_degree=1)
    r = CudaRenderer(s)
    r.set_blend_config(*cfg)
    v = _view(s, 0.3, 0.1, 0.8)
    full, small = Frame(), Frame()
    r.render(v, 131, 75, (0.2, 0.1, 0.0), full)
    r.render(v, 131, 75, (0.2, 0.1, 0.0), small, downsample=f)
    assert np.array_equal(small.pixels, oracle.downsample(full.pixels, f))
    r.close()


def _batch_setup():
    sc = [scenes.clusters(30_000, seed=51, sh_degree=0), scenes.clusters(60_000, seed=52, sh_degree=1),
          scenes.clusters(90_000, seed=53, sh_degree=3).to_fp16()]
    rends = [CudaRenderer(x) for x in sc]
    rng = np.random.default_rng(9)
    sizes = [(160, 96), (320, 192), (640, 360), (97, 53), (1280, 720), (33, 200)]
    views = []
    for i in range(14):
        k = i % 3
        src = sc[k] if k < 2 else scenes.clusters(90_000, seed=53, sh_degree=3)
        w, h = sizes[int(rng.integers(len(sizes)))]
        views.append(BatchView(k, _view(src, float(rng.uniform(0, 6.28)), float(rng.uniform(-0.5, 0.5)),
                                        float(rng.uniform(0.5, 1.5))), w, h,
                               tuple(float(x) for x in rng.uniform(0, 1, 3))))
    return sc, rends, views


def _single(rends, views, exact):
    out, stats = [], []
    for bv in views:
        r = rends[bv.scene]
        r.set_exact(exact)
        f = Frame()
        st = r.render(bv.view, bv.width, bv.height, bv.background, f, downsample=bv.downsample)
        out.append(f.pixels.copy())
        stats.append(st)
    return out, stats


def test_batch_matches_single_view_path():
    sc, rends, views = _batch_setup()
    want, want_st = _single(rends, views, exact=True)
    b = BatchRenderer(rends, views)
    b.set_exact(True)
    stats, ms = b.render()
    got = b.frames()
    for i in range(len(views)):
        assert np.array_equal(got[i], want[i]), f"view {i}: {np.sum(got[i] != want[i])} channels differ"
        assert stats[i].visible == want_st[i].visible and stats[i].overlaps == want_st[i].overlaps, i
    # A replay of the recorded graph repeats it.
    b.frames_dev.zero_()
    b.render()
    again = b.frames()
    for i in range(len(views)):
        assert np.array_equal(again[i], want[i]), f"replay view {i}"
    # The default blend agrees with the single-view default blend.
    fast, _ = _single(rends, views, exact=False)
    b.set_exact(False)
    b.render()
    got = b.frames()
    for i in range(len(views)):
        assert np.array_equal(got[i], fast[i]), f"fast view {i}"
    b.close()
    for r in rends:
        r.close()


def test_batch_configs_and_tuner():
    sc, rends, views = _batch_setup()
    want, _ = _single(rends, views, exact=True)
    b = BatchRenderer(rends, views)
    b.set_exact(True)
    for cfg in N.BLEND_CONFIGS:
        b.set_config(*cfg)
        assert b.config == cfg
        b.render()
        got = b.frames()
        for i in range(len(views)):
            assert np.array_equal(got[i], want[i]), f"{cfg} view {i}"
    res = b.autotune(reps=3)
    assert sorted(c for c, _ in res) == sorted(N.BLEND_CONFIGS)
    best = min(res, key=lambda x: x[1])[0]
    assert b.config == best
    assert all(ms > 0 for _, ms in res)
    b.render()
    got = b.frames()
    for i in range(len(views)):
        assert np.array_equal(got[i], want[i]), f"tuned view {i}"
    n0 = b.get_option(N.SPLAT_OPT_KERNEL_LAUNCHES)
    b.render()
    # project, count, column scan, ranges, scatter, long sort, blend; plus the
    # small and mid tile sorts unless the blend sorts them (16x16 tiles, 512 threads)
    want_launches = 7 if tuple(b.config) == (16, 16, 512) else 9
    assert b.get_option(N.SPLAT_OPT_KERNEL_LAUNCHES) - n0 == want_launches
    b.close()
    for r in rends:
        r.close()


def test_batch_downsample_and_validation(oracle):
    s = scenes.clusters(20_000, seed=61, sh_degree=2)
    r = CudaRenderer(s)
    v = _view(s, 1.0, 0.1, 0.9)
    full = Frame()
    r.render(v, 320, 180, (0.0, 0.0, 0.0), full)
    b = BatchRenderer([r], [BatchView(0, v, 320, 180, downsample=2), BatchView(0, v, 320, 180, downsample=4)])
    b.render()
    got = b.frames()
    assert np.array_equal(got[0], oracle.downsample(full.pixels, 2))
    assert np.array_equal(got[1], oracle.downsample(full.pixels, 4))
    with pytest.raises(N.SplatError):
        b.set_config(8, 8, 64)  # unsupported thread count
    with pytest.raises(N.SplatError):
        BatchRenderer([r], [BatchView(0, v, 320, 180, downsample=3)])  # 3 divides no tile shape
    b.close()
    r.close()
