"""The oracle pinned against the reference's own known answers and tests.

Each test cites the reference test it restates. These run on the CPU.
"""

import numpy as np
import pytest

from splat_b200 import OrbitCamera, UpAxis, View, synth
from tests import scenes


def xorshift(seed):
    # src/render/radix.rs:65-70
    seed ^= (seed << 13) & 0xFFFFFFFFFFFFFFFF
    seed ^= seed >> 7
    seed ^= (seed << 17) & 0xFFFFFFFFFFFFFFFF
    return seed


def test_fix_ties_orders_equal_depths_by_original_index(oracle):
    # src/render/cpu.rs:738-746
    orig = np.array([5, 3, 9, 0, 7, 1], np.uint32)
    k = lambda d, i: (d << 32) | i
    keys = np.array([k(1, 4), k(2, 0), k(2, 1), k(2, 2), k(3, 5), k(4, 3), k(4, 4)], np.uint64)
    want = np.array([k(1, 4), k(2, 1), k(2, 0), k(2, 2), k(3, 5), k(4, 3), k(4, 4)], np.uint64)
    assert np.array_equal(oracle.fix_ties(keys, orig), want)


@pytest.mark.parametrize("n", [0, 1, 2, 7, 192, 193, 1000, 5000, 70_000])
def test_sort_hi32_matches_stable_sort(oracle, n):
    # src/render/radix.rs:82-93
    def check(hi):
        seed = 0x9E3779B97F4A7C15 ^ n
        his = []
        for _ in range(n):
            seed = xorshift(seed)
            his.append(hi(seed))
        keys = (np.array(his, np.uint64) << np.uint64(32)) | np.arange(n, dtype=np.uint64)
        want = keys[np.argsort(keys >> np.uint64(32), kind="stable")]
        assert np.array_equal(oracle.sort_hi32(keys), want)

    check(lambda s: s & 0xFFFFFFFF)
    check(lambda s: s % 5)
    check(lambda s: int(np.float32(1.0 + (s % 1000) * np.float32(1e-3)).view(np.uint32)))
    check(lambda s: 42)


def test_sort_hi32_float_bits_order(oracle):
    # src/render/radix.rs:95-105
    seed = 7
    depths = []
    for _ in range(3000):
        seed = xorshift(seed)
        depths.append(np.float32(seed % 100_000) * np.float32(0.37) + np.float32(0.01))
    depths = np.array(depths, np.float32)
    keys = (depths.view(np.uint32).astype(np.uint64) << np.uint64(32)) | np.arange(3000, dtype=np.uint64)
    out = oracle.sort_hi32(keys)
    d = depths[(out & np.uint64(0xFFFFFFFF)).astype(np.int64)]
    assert np.all(d[:-1] <= d[1:])


def test_exp_neg_matches_exp(oracle):
    # src/render/simd.rs:338-354
    x = np.arange(-90.0, 0.0, 0.0137, dtype=np.float64).astype(np.float32)
    worst = 0.0
    for s in (1.0, 0.5, 0.1, 0.01):
        xi = (x * np.float32(s)).astype(np.float32)
        got = oracle.exp_neg(xi).astype(np.float64)
        want = np.exp(np.maximum(xi, np.float32(-87.0)).astype(np.float64))
        worst = max(worst, float(np.max(np.abs((got - want) / want))))
    assert worst < 5e-7
    assert np.all(oracle.exp_neg(np.zeros(4, np.float32)) == 1.0)


def test_downsample_known_answers(oracle):
    # src/term.rs:141-149
    src = np.array([[[0] * 3, [100] * 3], [[200] * 3, [100] * 3]], np.uint8)
    assert oracle.downsample(src, 2).tolist() == [[[100, 100, 100]]]

    # tests/term.rs:10-62
    def gradient(w, h):
        y, x = np.mgrid[0:h, 0:w]
        return np.stack([x % 256, y % 256, (x + y) % 256], -1).astype(np.uint8)

    d = oracle.downsample(gradient(7, 5), 2)
    assert d.shape == (2, 3, 3)
    assert d[0, 0].tolist() == [0, 0, 1]
    assert d[1, 2].tolist() == [(4 + 5 + 4 + 5) // 4, (2 + 2 + 3 + 3) // 4, (6 + 7 + 7 + 8) // 4]
    assert oracle.downsample(gradient(3, 3), 4).shape == (0, 0, 3)
    for f in (0, 1):
        assert np.array_equal(oracle.downsample(gradient(5, 4), f), gradient(5, 4))
    white = np.full((9, 9, 3), 255, np.uint8)
    for f in (2, 3, 4):
        d = oracle.downsample(white, f)
        assert d.shape[1] == 9 // f and np.all(d == 255)


def test_psnr_identical_is_infinite(oracle):
    # src/bench.rs:248-252
    f = np.zeros((4, 4, 3), np.uint8)
    assert np.isinf(oracle.psnr(f, f))


def test_covariance_known_answers(oracle):
    # src/scene.rs:289-302
    assert oracle.covariance([1, 2, 3], [0, 0, 0, 1]).tolist() == [1, 0, 0, 4, 0, 9]
    h = np.pi / 4
    c = oracle.covariance([1, 2, 3], [0, 0, np.sin(h), np.cos(h)])
    assert abs(c[0] - 4) < 1e-5 and abs(c[3] - 1) < 1e-5 and abs(c[1]) < 1e-5


def test_sh_identities(oracle):
    # src/sh.rs:79-91
    assert oracle.eval_rest(0, np.zeros(3), [1, 0, 0]).tolist() == [0, 0, 0]
    rest = np.array([[0, 0, 0], [1, 1, 1], [0, 0, 0]], np.float32)
    a = oracle.eval_rest(1, rest, [0, 0, 1])
    b = oracle.eval_rest(1, rest, [0, 0, -1])
    assert np.linalg.norm(a + b) < 1e-6 and a[0] > 0


def test_spread3_interleaves(oracle):
    # src/render/cpu.rs:338-346: bit i of v lands on bit 3i.
    for v in (0, 1, 2, 0x3FF, 0x155, 0x2AA):
        want = sum(((v >> i) & 1) << (3 * i) for i in range(10))
        assert oracle.spread3(v) == want


def view_at(eye):
    return View.looking_along_z(eye)


RED = (1.0, 0.0, 0.0)
BLUE = (0.0, 0.0, 1.0)


def both(oracle, s, v, w, h, bg):
    a, sa = oracle.render_naive(s, v, w, h, bg)
    c = oracle.CpuTiled(s)
    b, sb = c.render(v, w, h, bg)
    c.close()
    return (a, sa), (b, sb)


def test_semantic_image_tests(oracle):
    """tests/render.rs:78-187 on both CPU restatements."""
    s = scenes.splats([((0, 0, 5), 0.5, 1.0, RED)])
    for w, h in [(64, 64), (65, 33), (200, 100)]:
        for img, _ in both(oracle, s, view_at((0, 0, 0)), w, h, (0, 0, 0)):
            c = img[h // 2, w // 2]
            assert c[0] > 200 and c[1] < 10 and c[2] < 10
            for x, y in [(0, 0), (w - 1, 0), (0, h - 1), (w - 1, h - 1)]:
                assert img[y, x].tolist() == [0, 0, 0]
    for img, _ in both(oracle, s, view_at((0, 0, 0)), 64, 64, (0, 1, 0)):
        assert img[0, 0].tolist() == [0, 255, 0]
    behind = scenes.splats([((0, 0, -5), 0.5, 1.0, RED)])
    for img, st in both(oracle, behind, view_at((0, 0, 0)), 40, 30, (0.5, 0.5, 0.5)):
        assert st["visible"] == 0 and np.all(img == 128)
    off = scenes.splats([((500, 0, 5), 0.5, 1.0, RED), ((0, 0, 5), 0.5, 0.0, RED)])
    for img, _ in both(oracle, off, view_at((0, 0, 0)), 50, 50, (0.2, 0.4, 0.6)):
        assert np.all(img == img[0, 0])
    for img, _ in both(oracle, scenes.empty(), view_at((0, 0, 0)), 20, 10, (1, 1, 1)):
        assert np.all(img == 255)
    blue = ((0, 0, 4), 0.5, 1.0, BLUE)
    red = ((0, 0, 8), 1.0, 1.0, RED)
    for order in ([blue, red], [red, blue]):
        for img, _ in both(oracle, scenes.splats(order), view_at((0, 0, 0)), 64, 64, (0, 0, 0)):
            c = img[32, 32]
            assert c[2] > 200 and c[0] < 10
    tr = scenes.splats([((0, 0, 4), 0.5, 0.5, BLUE), ((0, 0, 8), 2.0, 1.0, RED)])
    for img, _ in both(oracle, tr, view_at((0, 0, 0)), 64, 64, (0, 0, 0)):
        assert img[32, 32, 0] > 40 and img[32, 32, 2] > 40
    right = scenes.splats([((1, 0, 5), 0.2, 1.0, RED)])
    for img, _ in both(oracle, right, view_at((0, 0, 0)), 100, 100, (0, 0, 0)):
        m = img[:, :, 0] > 100
        assert m[:, 50:].sum() > 0 and m[:, :50].sum() == 0


def test_cpu_agrees_with_naive_on_reference_scenes(oracle):
    """tests/render.rs:45-76 (>= 45 dB between cpu and cpu-naive)."""
    for s, sizes in [(scenes.cube(), [(1, 1), (17, 9), (64, 48), (333, 77)]), (scenes.shballs(), [(97, 53)])]:
        c, r = s.bounds()
        cpu = oracle.CpuTiled(s)
        for up, yaw, pitch in [(UpAxis.NEG_Y, 0.37, 0.26), (UpAxis.POS_Y, 4.0, 0.9), (UpAxis.POS_Z, 2.0, 0.1)]:
            cam = OrbitCamera.new(c, r, up)
            cam.rotate(yaw, np.float32(pitch) - cam.pitch)
            v = cam.view()
            for w, h in sizes:
                a, _ = cpu.render(v, w, h, (0.1, 0.2, 0.3))
                b, _ = oracle.render_naive(s, v, w, h, (0.1, 0.2, 0.3))
                assert oracle.psnr(a, b) >= 45.0
        cpu.close()


def test_cpu_is_deterministic_across_thread_counts(oracle):
    s = synth.cluster_scene(5000, seed=3)
    v = synth.orbit_camera(s).view()
    imgs = []
    for t in (1, 3, 8):
        c = oracle.CpuTiled(s, threads=t)
        imgs.append(c.render(v, 160, 90)[0])
        c.close()
    assert all(np.array_equal(imgs[0], i) for i in imgs[1:])


def test_zero_size_and_pixel_limit(oracle):
    s = scenes.cube()
    v = view_at((0, 0, -5))
    for w, h in [(0, 0), (64, 0), (0, 64)]:
        img, st = oracle.render_naive(s, v, w, h)
        assert img.size == 0 and st["visible"] == 0
    with pytest.raises(ValueError, match="pixel limit"):
        oracle.render_naive(s, v, 16385, 1)


def test_bin_sort_orders_by_tile_depth_index(oracle):
    # Three splats sharing tile 0; two with equal depth keep index order.
    x = np.array([5, 5, 5, 40], np.float32)
    y = np.array([5, 5, 5, 5], np.float32)
    e = np.array([2, 2, 2, 2], np.float32)
    d = np.array([3.0, 2.0, 3.0, 1.0], np.float32)
    keys, vals, ranges = oracle.bin_sort(x, y, e, e, d, np.ones(4, bool), 48, 16)
    assert vals.tolist() == [1, 0, 2, 3]
    assert ranges.tolist() == [[0, 3], [0, 0], [3, 4]]
    assert (keys >> np.uint64(32)).tolist() == [0, 0, 0, 2]
