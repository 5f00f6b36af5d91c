"""ORACLE — test infrastructure only.

Restatement of the terminal mapping of ``src/term.rs``: ``rgb_to_ansi256``
(``term.rs:48-72``), ``ColorMode::color`` (``term.rs:39-45``) and the cells
the ``HalfBlockImage`` widget draws (``term.rs:109-130``), for checking the
device's ``splat_cuda_render_cells``. Only tests import it.
"""

from __future__ import annotations

import numpy as np

LEVELS = (0, 95, 135, 175, 215, 255)


def rgb_to_ansi256(c) -> int:
    """Nearest xterm-256 colour, cube or gray ramp (term.rs:48-72)."""
    r, g, b = (int(v) for v in c)

    def cube_idx(v):
        if v < 48:
            return 0
        if v < 115:
            return 1
        return min((v - 35) // 40, 5)

    ri, gi, bi = cube_idx(r), cube_idx(g), cube_idx(b)
    cube = (LEVELS[ri], LEVELS[gi], LEVELS[bi])
    avg = (r + g + b) // 3
    gray_idx = min(max(int((avg - 3) / 10), 0), 23)  # Rust's truncating division
    gray = 8 + gray_idx * 10

    def dist(a):
        return sum((a[k] - (r, g, b)[k]) ** 2 for k in range(3))

    return 232 + gray_idx if dist((gray,) * 3) < dist(cube) else 16 + 36 * ri + 6 * gi + bi


def palette(i: int):
    if i >= 232:
        g = 8 + (i - 232) * 10
        return (g, g, g)
    i -= 16
    return (LEVELS[i // 36], LEVELS[(i // 6) % 6], LEVELS[i % 6])


def cells(img, mode: str):
    """The widget's cells of an (h, w, 3) u8 frame: (h // 2, w, 6) truecolor
    (fg RGB, bg RGB) or (h // 2, w, 2) ansi256 indices."""
    img = np.asarray(img, np.uint8)
    rows, cols = img.shape[0] // 2, img.shape[1]
    top, bot = img[0:2 * rows:2], img[1:2 * rows:2]
    if mode == "truecolor":
        return np.concatenate([top, bot], axis=2)
    lut = {}
    out = np.zeros((rows, cols, 2), np.uint8)
    for y in range(rows):
        for x in range(cols):
            for k, px in ((0, top[y, x]), (1, bot[y, x])):
                key = tuple(int(v) for v in px)
                if key not in lut:
                    lut[key] = rgb_to_ansi256(key)
                out[y, x, k] = lut[key]
    return out
