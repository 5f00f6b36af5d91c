"""The closed form behind the ellipse pairs (ellipse_skips in
splat_b200/csrc/common.cuh) and the blend's warp-block masks (block_mask in
splat_b200/csrc/blend.cu), checked in float64 on the CPU.

For the ellipse Q(dx, dy) = a dx^2 + 2 b dx dy + c dy^2 <= K and a band of
rows dy in [lo, hi], the kernels take the ellipse's x range inside the band
as [L(yl), U(yr)] with U/L(dy) = (-b dy +/- sqrt(a K - det dy^2)) / a and
yr / yl the rightmost / leftmost points of the ellipse (dy = -/+ b sqrt(K c /
det) / c) clamped into the band. The test compares that range with a dense
sampling of the band and checks that the rectangles it leaves out miss the
ellipse (exact minimum of Q over a rectangle), for round, tilted and very
thin ellipses."""

import numpy as np


def band_range(a, b, c, K, lo, hi):
    """[xl, xu] of the ellipse inside the band lo <= dy <= hi (None when the
    band misses the ellipse), as the kernels compute it."""
    det = a * c - b * b
    ey = np.sqrt(K * a / det)
    if hi < -ey or lo > ey:
        return None
    lo, hi = max(lo, -ey), min(hi, ey)
    xm = np.sqrt(K * c / det)
    dyr = -b * xm / c
    yr, yl = min(max(dyr, lo), hi), min(max(-dyr, lo), hi)
    U = (-b * yr + np.sqrt(max(a * K - det * yr * yr, 0.0))) / a
    L = (-b * yl - np.sqrt(max(a * K - det * yl * yl, 0.0))) / a
    return L, U


def rect_min_q(a, b, c, x0, x1, y0, y1):
    """The minimum of Q over the rectangle [x0, x1] x [y0, y1] (offsets from
    the centre)."""
    if x0 <= 0 <= x1 and y0 <= 0 <= y1:
        return 0.0

    def q(dx, dy):
        return a * dx * dx + 2 * b * dx * dy + c * dy * dy

    cands = []
    for dx in (x0, x1):
        cands.append(q(dx, min(max(-b * dx / c, y0), y1)))
    for dy in (y0, y1):
        cands.append(q(min(max(-b * dy / a, x0), x1), dy))
    return min(cands)


def random_ellipses(rng, n):
    out = []
    for i in range(n):
        s1 = 10 ** rng.uniform(-0.5, 1.5)
        s2 = s1 * (10 ** rng.uniform(-2.5, 0.0) if i % 3 else 1.0)  # every third round
        th = rng.uniform(0, np.pi)
        R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
        cov = R @ np.diag([s1 * s1 + 0.3, s2 * s2 + 0.3]) @ R.T  # the projection's dilation
        con = np.linalg.inv(cov)
        K = 2 * np.log(255 * rng.uniform(0.01, 1.0))
        out.append((con[0, 0], con[0, 1], con[1, 1], K))
    return out


def test_band_range_matches_dense_sampling():
    rng = np.random.default_rng(7)
    for a, b, c, K in random_ellipses(rng, 300):
        ey = np.sqrt(K * a / (a * c - b * b))
        lo = rng.uniform(-1.5 * ey, 1.2 * ey)
        hi = lo + rng.uniform(0.0, 2.0 * ey)
        r = band_range(a, b, c, K, lo, hi)
        dys = np.linspace(max(lo, -ey), min(hi, ey), 4001)
        if r is None:
            assert hi < -ey or lo > ey
            continue
        det = a * c - b * b
        disc = np.maximum(a * K - det * dys * dys, 0.0)
        u = ((-b * dys + np.sqrt(disc)) / a).max()
        l_ = ((-b * dys - np.sqrt(disc)) / a).min()
        scale = np.sqrt(K * c / det)
        assert r[1] >= u - 1e-9 * scale and r[1] <= u + 1e-3 * scale
        assert r[0] <= l_ + 1e-9 * scale and r[0] >= l_ - 1e-3 * scale


def test_left_out_tiles_miss_the_ellipse():
    """Tiles of 16 x 16 pixels around each ellipse: a tile whose
    pixel-centre columns miss the band's range (the kernels' rule) has
    min Q > K over its pixel-centre rectangle; a kept tile may still miss
    (the rule is per row band), but no reached tile is dropped."""
    rng = np.random.default_rng(11)
    dropped = kept_reached = 0
    for a, b, c, K in random_ellipses(rng, 200):
        x, y = rng.uniform(0, 16, 2)  # the centre inside tile (0, 0)
        det = a * c - b * b
        ex, ey = np.sqrt(K * c / det), np.sqrt(K * a / det)
        for ty in range(int(np.floor((y - ey) / 16)), int(np.floor((y + ey) / 16)) + 1):
            y0, y1 = 16 * ty + 0.5 - y, 16 * ty + 15.5 - y
            r = band_range(a, b, c, K, y0, y1)
            for tx in range(int(np.floor((x - ex) / 16)), int(np.floor((x + ex) / 16)) + 1):
                x0, x1 = 16 * tx + 0.5 - x, 16 * tx + 15.5 - x
                reach = rect_min_q(a, b, c, x0, x1, y0, y1) <= K
                keep = r is not None and x1 >= r[0] and x0 <= r[1]
                if reach:
                    assert keep, (a, b, c, K, tx, ty)
                    kept_reached += 1
                else:
                    dropped += not keep
    assert kept_reached > 0 and dropped > 0
