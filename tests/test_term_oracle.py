"""The terminal mapping's oracle (oracle/term_oracle.py) against the
reference's own tests (src/term.rs:131-175, tests/term.rs:64-140)."""

import numpy as np

from oracle import term_oracle as T


def test_ansi256_extremes():
    assert T.rgb_to_ansi256((0, 0, 0)) == 16
    assert T.rgb_to_ansi256((255, 255, 255)) == 231
    assert T.rgb_to_ansi256((255, 0, 0)) == 196
    assert 232 <= T.rgb_to_ansi256((128, 128, 128)) <= 255


def test_ansi256_exact_cube_colors_map_exactly():
    for r in T.LEVELS:
        for g in T.LEVELS:
            for b in T.LEVELS:
                assert T.palette(T.rgb_to_ansi256((r, g, b))) == (r, g, b)


def test_ansi256_gray_ramp_exact():
    for i in range(232, 256):
        g = T.palette(i)[0]
        assert T.rgb_to_ansi256((g, g, g)) == i


def test_ansi256_is_nearest_within_reason():
    pal = np.array([T.palette(i) for i in range(16, 256)])
    for r in range(0, 256, 7):
        for g in range(0, 256, 11):
            for b in range(0, 256, 13):
                idx = T.rgb_to_ansi256((r, g, b))
                assert idx >= 16
                d = ((pal - np.array([r, g, b])) ** 2).sum(1)
                got = sum((p - c) ** 2 for p, c in zip(T.palette(idx), (r, g, b)))
                assert got - d.min() <= 1500


def test_widget_draws_half_blocks():
    f = np.array([[[255, 0, 0], [0, 255, 0]], [[0, 0, 255], [9, 9, 9]]], np.uint8)
    c = T.cells(f, "truecolor")
    assert c.shape == (1, 2, 6)
    assert list(c[0, 0]) == [255, 0, 0, 0, 0, 255]
    assert list(T.cells(f, "ansi256")[0, 0]) == [196, 21]
