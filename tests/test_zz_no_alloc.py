"""splat_cuda_sort_tile_noalloc, the entry point for callers that cannot
allocate device memory (their device memory belongs to another allocator, or
they must not allocate while they run). It sorts one tile's pairs using a
static device array as its only scratch.

Its output is checked against the existing entry points: a frame rendered
through splat_cuda_render with debug capture, whose per-tile pair order
splat_cuda_debug_dump reports. The same pairs, shuffled, go through the
no-allocation sort twice in a row (two tiles, the scratch array reused) and
must come back in exactly that order (integer data: bit-exact). This file is
collected last so that a failure here stops a `-x` run only after every
other test has run.
"""

import ctypes

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _sorted_tiles():
    s = scenes.clusters(20_000, seed=7, sh_degree=3)
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.zoom(0.6)
    v = cam.view()
    rend = CudaRenderer(s)
    rend.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    rend.render(v, 640, 360, (0.0, 0.0, 0.0), Frame())
    d = rend.debug_dump(640, 360)
    rend.close()
    words = ((d["keys"] & np.uint64(0xFFFFFFFF)) << np.uint64(32)) | d["values"].astype(np.uint64)
    lengths = d["ranges"][:, 1].astype(np.int64) - d["ranges"][:, 0].astype(np.int64)
    return words, d["ranges"], lengths


def test_no_alloc_sort_matches_render_order():
    import torch

    words, ranges, lengths = _sorted_tiles()
    order = np.argsort(-lengths, kind="stable")
    tiles = [int(order[0]), int(order[len(order) // 8])]  # the longest tile and a shorter one
    assert lengths[tiles[0]] > 1 and lengths[tiles[1]] > 1
    lib = N.lib()
    rng = np.random.default_rng(3)
    for t in tiles:  # two calls in a row share the scratch array
        b, e = int(ranges[t, 0]), int(ranges[t, 1])
        want = words[b:e].copy()
        shuffled = want[rng.permutation(len(want))]
        dev = torch.from_numpy(shuffled.view(np.int64)).cuda()
        torch.cuda.synchronize()
        rc = lib.splat_cuda_sort_tile_noalloc(ctypes.c_void_p(dev.data_ptr()), len(want),
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == N.SPLAT_OK
        torch.cuda.synchronize()
        got = dev.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), f"tile {t}: {np.sum(got != want)} of {len(want)} pairs out of order"


def _words(rng, n, depth_levels):
    """n distinct pair words: depth bits from `depth_levels` distinct positive
    floats (few levels: long runs of equal depth), splat indices distinct."""
    depths = np.sort(rng.uniform(0.5, 40.0, depth_levels).astype(np.float32)).view(np.uint32)
    d = depths[rng.integers(0, depth_levels, n)].astype(np.uint64)
    idx = rng.choice(1 << 24, n, replace=False).astype(np.uint64)
    return (d << np.uint64(32)) | idx


@pytest.mark.parametrize("n,levels", [(4097, 3), (300_000, 1000), (300_000, 1), (MAX_PAIRS, 50_000),
                                      (MAX_PAIRS, 2)])
def test_no_alloc_sort_matches_full_word_order(n, levels):
    """Tiles longer than one shared-memory chunk (the carried digit starts),
    depth bytes that do not vary (skipped passes), the size limit, and runs
    of equal depth up to the whole tile: the result is the words in
    ascending order (depth bits, then splat index), equal to a sort of the
    words on the host; three calls in a row reuse the scratch array."""
    import torch

    lib = N.lib()
    rng = np.random.default_rng(n + levels)
    for call in range(3):
        words = _words(rng, n, levels)
        dev = torch.from_numpy(words.view(np.int64)).cuda()
        rc = lib.splat_cuda_sort_tile_noalloc(ctypes.c_void_p(dev.data_ptr()), n,
                                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == N.SPLAT_OK
        torch.cuda.synchronize()
        got = dev.cpu().numpy().view(np.uint64)
        want = np.sort(words)
        assert np.array_equal(got, want), f"call {call}: {np.sum(got != want)} of {n} words out of order"


def test_no_alloc_sort_rejects_more_than_its_scratch():
    rc = N.lib().splat_cuda_sort_tile_noalloc(ctypes.c_void_p(0), MAX_PAIRS + 1, None)
    assert rc == N.SPLAT_ERR_INVALID_ARG
