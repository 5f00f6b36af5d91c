"""The blend's evaluation count (SPLAT_OPT_COUNT_EVALS / SPLAT_OPT_BLEND_EVALS):
the pixel/splat evaluations the default blend performs after early
termination, the unit of its arithmetic work. Counting leaves the image
unchanged; known answers on small scenes bound it from both sides."""

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


def _axis_view():
    return View(np.zeros(3, f32), np.array([1, 0, 0], f32), np.array([0, 1, 0], f32), np.array([0, 0, 1], f32),
                f32(1.0), f32(0.01))


def test_one_screen_filling_splat_is_evaluated_once_per_pixel():
    s = Scene()
    s.push((0.0, 0.0, 1.0), (50.0, 50.0, 50.0), (0, 0, 0, 1), 0.3, (1.0, 0.5, 0.0))
    s = s.finalize()
    r = CudaRenderer(s)
    try:
        r.set_option(N.SPLAT_OPT_COUNT_EVALS, 1)
        r.render(_axis_view(), 64, 48, (0.0, 0.0, 0.0), Frame())
        assert r.get_option(N.SPLAT_OPT_BLEND_EVALS) == 64 * 48
    finally:
        r.close()


def test_counting_leaves_the_image_and_bounds_hold():
    s = scenes.clusters(20_000, seed=7, sh_degree=3)
    from splat_b200 import OrbitCamera, UpAxis

    c, rad = s.bounds()
    v = OrbitCamera.new(c, rad, UpAxis.NEG_Y).view()
    r = CudaRenderer(s)
    try:
        a, b = Frame(), Frame()
        st = r.render(v, 640, 360, (0.1, 0.2, 0.3), a)
        assert r.get_option(N.SPLAT_OPT_BLEND_EVALS) == 0
        r.set_option(N.SPLAT_OPT_COUNT_EVALS, 1)
        r.render(v, 640, 360, (0.1, 0.2, 0.3), b)
        e = r.get_option(N.SPLAT_OPT_BLEND_EVALS)
        assert np.array_equal(a.pixels, b.pixels)
        # Every pixel evaluates at most every pair of its tile (+1: pairs of
        # two splats are evaluated together); at least the first splat of
        # each non-empty tile is evaluated by the pixels of its block.
        assert 0 < e <= st.overlaps * 256 + 640 * 360
        r.set_option(N.SPLAT_OPT_COUNT_EVALS, 0)
        r.render(v, 640, 360, (0.1, 0.2, 0.3), b)
        assert r.get_option(N.SPLAT_OPT_BLEND_EVALS) == 0
    finally:
        r.close()
