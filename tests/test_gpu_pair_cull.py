"""Pairs only where the splat reaches the tile (the default) against the
reference's pairs, every tile of the pixel bbox (SPLAT_OPT_BBOX_PAIRS).

* The images are the same, byte for byte, in the default and the exact
  blend (so the exact blend still equals the cpu backend), for FP32 and
  FP16 storage, thin needles, three tile shapes, windows of rows.
* The pairs drawn are a subset of the bbox pairs, tile by tile in the same
  order, and every pair left out belongs to a tile whose pixel centres all
  lie outside the splat's alpha = 1/255 ellipse (checked in float64 from the
  device's own projection and the scene's opacities).
* At the 1.2M-splat 1080p workload the rule leaves out about 15 % of the
  pairs.
"""

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200 import synth
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu


def _views(s, n=3):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    out = [cam.view()]
    for i in range(n - 1):
        cam.rotate(1.3, 0.0)
        cam.zoom(0.55 if i % 2 == 0 else 1.6)
        out.append(cam.view())
    return out


def _frame(r, view, w, h, bbox, exact=False, bg=(0.1, 0.2, 0.3)):
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, int(bbox))
    r.set_exact(exact)
    f = Frame()
    st = r.render(view, w, h, bg, f)
    return f.pixels.copy(), st


@pytest.mark.parametrize("name", ["clusters", "needles", "galaxy"])
@pytest.mark.parametrize("blend", [(16, 16, 512), (8, 8, 256), (32, 16, 512)])
def test_images_do_not_change(name, blend):
    s = {"clusters": lambda: scenes.clusters(20_000, seed=7, sh_degree=3),
         "needles": lambda: scenes.needles(20_000, seed=5),
         "galaxy": scenes.galaxy}[name]()
    r = CudaRenderer(s)
    r.set_blend_config(*blend)
    try:
        for v in _views(s):
            for exact in (False, True):
                a, sa = _frame(r, v, 640, 360, bbox=True, exact=exact)
                b, sb = _frame(r, v, 640, 360, bbox=False, exact=exact)
                assert np.array_equal(a, b), f"{name} {blend} exact={exact}: {np.sum(a != b)} channels differ"
                assert sb.overlaps <= sa.overlaps and sb.visible == sa.visible
            rows_a = r.render_rows(v, 640, 360, (0.1, 0.2, 0.3), 37, 200)
            assert np.array_equal(rows_a, b[37:237])
    finally:
        r.close()


def test_fp16_images_do_not_change():
    s = scenes.clusters(20_000, seed=17, sh_degree=3)
    r = CudaRenderer(s.to_fp16())
    try:
        for v in _views(s):
            a, sa = _frame(r, v, 512, 288, bbox=True)
            b, sb = _frame(r, v, 512, 288, bbox=False)
            assert np.array_equal(a, b)
            assert sb.overlaps < sa.overlaps
    finally:
        r.close()


def _pairs(r, view, w, h, bbox):
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, int(bbox))
    r.render(view, w, h, (0.0, 0.0, 0.0), Frame())
    d = r.debug_dump(w, h)
    return d


@pytest.mark.parametrize("name", ["clusters", "needles"])
def test_left_out_pairs_miss_the_ellipse(name):
    s = scenes.clusters(20_000, seed=7, sh_degree=3) if name == "clusters" else scenes.needles(20_000, seed=5)
    w, h = 640, 360
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    try:
        for v in _views(s):
            full = _pairs(r, v, w, h, bbox=True)
            cut = _pairs(r, v, w, h, bbox=False)
            tiles_x = (w + 15) // 16
            kept = 0
            gone_t, gone_i = [], []
            for t in range(len(full["ranges"])):
                fa, fb = full["ranges"][t]
                ca, cb = cut["ranges"][t]
                fk, fv = full["keys"][fa:fb], full["values"][fa:fb]
                cv = cut["values"][ca:cb]
                # the tile's pairs: a subsequence of its bbox pairs (same order)
                idx = {int(x): j for j, x in enumerate(fv)}
                assert all(int(x) in idx for x in cv), f"tile {t}: a pair outside the bbox pairs"
                js = [idx[int(x)] for x in cv]
                assert js == sorted(js), f"tile {t}: not in the bbox pairs' order"
                assert np.array_equal(cut["keys"][ca:cb], fk[js]), f"tile {t}: keys differ"
                kept += len(cv)
                left = np.setdiff1d(fv, cv)
                gone_t += [t] * len(left)
                gone_i += list(left)
            assert kept == len(cut["keys"]) and kept <= len(full["keys"])
            if not gone_i:
                continue
            # every left-out pair: the tile's pixel-centre rectangle misses the ellipse
            p = cut["proj"].astype(np.float64)
            gi = np.array(gone_i, np.int64)
            gt = np.array(gone_t, np.int64)
            x, y, a, b, c = p[gi, 0], p[gi, 1], p[gi, 5], p[gi, 6], p[gi, 7]
            K = 2.0 * np.log(255.0 * s.opacities[gi].astype(np.float64))
            tx, ty = gt % tiles_x, gt // tiles_x
            X0, X1 = 16 * tx + 0.5 - x, 16 * tx + 15.5 - x
            Y0, Y1 = 16 * ty + 0.5 - y, 16 * ty + 15.5 - y

            def q(dx, dy):
                return a * dx * dx + 2 * b * dx * dy + c * dy * dy

            m = np.minimum.reduce([q(X0, np.clip(-b * X0 / c, Y0, Y1)), q(X1, np.clip(-b * X1 / c, Y0, Y1)),
                                   q(np.clip(-b * Y0 / a, X0, X1), Y0), q(np.clip(-b * Y1 / a, X0, X1), Y1)])
            inside = (X0 <= 0) & (X1 >= 0) & (Y0 <= 0) & (Y1 >= 0)
            assert not inside.any()
            assert np.all(m > K * (1.0 - 1e-5)), f"a left-out tile is reached: min Q / K = {np.min(m / K)}"
    finally:
        r.close()


def test_headline_workload_leaves_out_a_seventh_of_the_pairs():
    scene = synth.cluster_scene(1_200_000, seed=0x5EED0001, sh_degree=3)
    cam = synth.orbit_camera(scene)
    home, _, timed = synth.orbit_views(cam, 40, 5)
    r = CudaRenderer(scene)
    try:
        for v in (home, timed[10]):
            a, sa = _frame(r, v, 1920, 1080, bbox=True, bg=(0.0, 0.0, 0.0))
            b, sb = _frame(r, v, 1920, 1080, bbox=False, bg=(0.0, 0.0, 0.0))
            assert np.array_equal(a, b)
            assert 0.75 * sa.overlaps < sb.overlaps < 0.95 * sa.overlaps, (sb.overlaps, sa.overlaps)
    finally:
        r.close()
