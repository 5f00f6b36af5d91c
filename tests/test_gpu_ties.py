"""Depth ties: pairs of one tile that share the depth bits are ordered by
splat index (the reference's sort_hi32 + fix_ties, src/render/radix.rs:13-57,
src/render/cpu.rs:396-414), and the cost of ordering them stays linear.

The scene puts every splat on one of two planes facing the camera, so each
tile's pairs form at most two runs of equal depth: up to ~19k pairs in the
long tiles (more than 4096 pairs: chunked LSD passes in global memory), and
runs far beyond the 32 items one thread orders in the mid (513-4096 pairs)
and warp (up to 512 pairs) sorts, which then sort the whole tile by the full
word. Gates: keys, values and ranges bit-identical to the oracle's
recomputation; the exact-blend image identical to the oracle `cpu` backend;
the default blend >= 60 dB / <= 2/255; the binning + sort stage of the frame
well under the time a quadratic ordering of the runs would take.
"""

import numpy as np
import pytest

from splat_b200 import Frame, View
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu

W, H = 320, 240


@pytest.fixture(scope="module")
def planes(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return scenes.planes()


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 16)])
def test_equal_depth_runs_order_by_splat_index(oracle, planes, tile):
    s = planes
    v = View.looking_along_z([0.0, 0.0, 0.0])
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    r.set_blend_config(tile[0], tile[1], 256)
    cpu = oracle.CpuTiled(s)
    try:
        f = Frame()
        r.set_exact(True)
        r.render(v, W, H, (0.1, 0.2, 0.3), f)
        st = r.render(v, W, H, (0.1, 0.2, 0.3), f)  # the second frame: buffers sized, kernels loaded
        d = r.debug_dump(W, H)
        pr = d["proj"]
        assert len(np.unique(pr[d["visible"], 4])) == 2, "every splat should lie on one of two depths"
        keys, vals, ranges = oracle.bin_sort(pr[:, 0], pr[:, 1], pr[:, 2], pr[:, 3], pr[:, 4], d["visible"], W, H,
                                             tile=tile)
        lengths = ranges[:, 1].astype(np.int64) - ranges[:, 0].astype(np.int64)
        if tile == (16, 16):
            assert (lengths > 4096).sum() > 10 and ((lengths > 512) & (lengths <= 4096)).sum() > 10
            assert ((lengths > 64) & (lengths <= 512)).sum() > 10
        assert np.array_equal(d["ranges"], ranges), "ranges differ"
        assert np.array_equal(d["keys"], keys), f"{np.sum(d['keys'] != keys)} keys differ"
        assert np.array_equal(d["values"], vals), f"{np.sum(d['values'] != vals)} values differ"
        assert st.sort_ms < 20.0, f"binning + sorts took {st.sort_ms:.2f} ms"
        want, _ = cpu.render(v, W, H, (0.1, 0.2, 0.3))
        assert np.array_equal(f.pixels, want), f"exact blend differs in {np.sum(f.pixels != want)} channels"
        r.set_exact(False)
        r.render(v, W, H, (0.1, 0.2, 0.3), f)
        p = oracle.psnr(f.pixels, want)
        err = int(np.max(np.abs(f.pixels.astype(int) - want.astype(int))))
        assert p >= 60.0 and err <= 2, f"psnr {p:.2f} max err {err}"
    finally:
        cpu.close()
        r.close()
