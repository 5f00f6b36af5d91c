"""ORACLE — test infrastructure only.

Independent numpy (float64) restatement of the learned-colour MLP that the
sm_100a library trains and evaluates: the forward pass, the backward pass of
the mean-squared-error loss, Adam, the per-epoch sample shuffle, the
Fibonacci-sphere directions and the exact SH targets they are trained on.
Only tests import it, as the checker.

There is no reference implementation of this part (the reference evaluates
degree-3 SH per splat, ``src/sh.rs:39-64``), so the restatement is pinned
two ways: ``eval_rest`` against the C++ restatement of ``sh::eval_rest``
(``oracle.eval_rest``), and the backward pass against central finite
differences of the forward pass (``tests/test_mlp_oracle.py``).

fp16 emulation: with ``emulate=True`` values are rounded to binary16 at the
points where the device stores them as tensor-core operands (the input row,
the parameters, h1, h2, dz3, dz2, dz1); accumulation stays float64.
"""

from __future__ import annotations

import numpy as np

LATENT = 16
IN = 32
HIDDEN = 64
OUT = 16
BIAS_COL = 19
W1, W2, B2, W3, B3 = 0, 2048, 6144, 6208, 7232
PARAMS = 7248
LOSS_SCALE = 128.0

# src/sh.rs:5-22
SH_C1 = 0.4886025
SH_C2 = (1.0925485, -1.0925485, 0.31539157, -1.0925485, 0.54627424)
SH_C3 = (-0.5900436, 2.8906114, -0.4570458, 0.37317633, -0.4570458, 1.4453057, -0.5900436)

M64 = (1 << 64) - 1


def f16(a):
    """Round to binary16 (nearest even) and widen back to float64."""
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def unpack(params):
    p = np.asarray(params, np.float64)
    return (p[W1:W2].reshape(HIDDEN, IN), p[W2:B2].reshape(HIDDEN, HIDDEN), p[B2:W3], p[W3:B3].reshape(OUT, HIDDEN),
            p[B3:PARAMS])


def pack(w1, w2, b2, w3, b3):
    return np.concatenate([w1.ravel(), w2.ravel(), b2.ravel(), w3.ravel(), b3.ravel()])


def eval_rest(degree, rest, d):
    """sh::eval_rest (src/sh.rs:39-64), vectorised: rest (n, per, 3), d (n, 3)."""
    rest = np.asarray(rest, np.float64)
    x, y, z = (np.asarray(d, np.float64)[:, k:k + 1] for k in range(3))
    out = np.zeros((len(rest), 3))
    if degree >= 1:
        out += SH_C1 * ((-y) * rest[:, 0] + z * rest[:, 1] - x * rest[:, 2])
    if degree >= 2:
        xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
        b = [SH_C2[0] * xy, SH_C2[1] * yz, SH_C2[2] * (2 * zz - xx - yy), SH_C2[3] * xz, SH_C2[4] * (xx - yy)]
        for k in range(5):
            out += b[k] * rest[:, 3 + k]
        if degree >= 3:
            b = [SH_C3[0] * y * (3 * xx - yy), SH_C3[1] * xy * z, SH_C3[2] * y * (4 * zz - xx - yy),
                 SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy), SH_C3[4] * x * (4 * zz - xx - yy),
                 SH_C3[5] * z * (xx - yy), SH_C3[6] * x * (xx - 3 * yy)]
            for k in range(7):
                out += b[k] * rest[:, 8 + k]
    return out


def sh_targets(colors, sh_rest, degree, d):
    """Training targets: base colour + eval_rest at d, clamped to [0, 1]."""
    c = np.asarray(colors, np.float64) + (eval_rest(degree, sh_rest, d) if degree else 0.0)
    return np.clip(c, 0.0, 1.0)


def fibonacci_dirs(n):
    """Unit directions of a Fibonacci sphere (the construction of src/gen.rs:213-219), f32."""
    i = np.arange(n, dtype=np.float64)
    y = 1.0 - 2.0 * (i + 0.5) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - y * y))
    th = np.pi * (3.0 - np.sqrt(5.0)) * i
    return np.stack([r * np.cos(th), y, r * np.sin(th)], 1).astype(np.float32)


def _mul(a, b):
    return (a * np.uint64(b)) & np.uint64(M64)


def shuffle_hash(x, key, bits):
    x = np.asarray(x, np.uint64)
    mask = np.uint64((1 << bits) - 1)
    s = np.uint64(bits // 2 + 1)
    x = (x ^ np.uint64(key & M64)) & mask
    x ^= x >> s
    x = _mul(x, 0x9E3779B97F4A7C15) & mask
    x ^= x >> s
    x = _mul(x, 0xC2B2AE3D27D4EB4F) & mask
    x ^= x >> s
    x = _mul(x, 0x165667B19E3779F9) & mask
    x ^= x >> s
    return x


def shuffle_index(i, m, key, bits):
    """The bijective shuffle of [0, m): hash, cycle-walked back into range."""
    i = np.asarray(i, np.uint64)
    x = shuffle_hash(i, key, bits)
    for _ in range(4096):
        out = x >= np.uint64(m)
        if not out.any():
            break
        x = np.where(out, shuffle_hash(x, key, bits), x)
    return np.where(x < np.uint64(m), x, i)


def epoch_key(seed, epoch):
    return (seed * 0x9E3779B97F4A7C15 + epoch * 0xD1B54A32D192ED03 + 1) & M64


def step_samples(step, n, n_dirs, batch, seed):
    """(splat, direction) indices of one step's active samples."""
    samples = n * n_dirs
    spe = (samples + batch - 1) // batch
    bits = 1
    while (1 << bits) < samples:
        bits += 1
    k = step % spe
    base = k * batch
    active = min(batch, samples - base)
    p = shuffle_index(np.arange(base, base + active, dtype=np.uint64), samples, epoch_key(seed, step // spe), bits)
    return (p // np.uint64(n_dirs)).astype(np.int64), (p % np.uint64(n_dirs)).astype(np.int64)


def forward(params, latents, dirs, emulate=True):
    """latents (B, 16), dirs (B, 3) -> dict with x, z1, h1, z2, h2, z3, y."""
    r = f16 if emulate else (lambda a: np.asarray(a, np.float64))
    w1, w2, b2, w3, b3 = (r(a) for a in unpack(params))
    b = len(latents)
    x = np.zeros((b, IN))
    x[:, :LATENT] = r(latents)
    x[:, LATENT:LATENT + 3] = r(dirs)
    x[:, BIAS_COL] = 1.0
    z1 = x @ w1.T
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ w2.T + b2
    h2 = r(np.maximum(z2, 0.0))
    z3 = h2 @ w3.T + b3
    y = 1.0 / (1.0 + np.exp(-z3[:, :3]))
    return {"x": x, "z1": z1, "h1": h1, "z2": z2, "h2": h2, "z3": z3, "y": y, "w": (w1, w2, b2, w3, b3)}


def loss(y, targets):
    return float(np.mean((y - targets) ** 2))


def backward(params, latents, dirs, targets, emulate=True):
    """Gradients of the mean squared error: (loss, y, d params, d latents)."""
    r = f16 if emulate else (lambda a: np.asarray(a, np.float64))
    f = forward(params, latents, dirs, emulate)
    w1, w2, b2, w3, b3 = f["w"]
    y, t = f["y"], np.asarray(targets, np.float64)
    b = len(y)
    s = LOSS_SCALE if emulate else 1.0
    dz3 = np.zeros((b, OUT))
    dz3[:, :3] = r(s * (2.0 / 3.0) * (y - t) * y * (1.0 - y))
    dh2 = dz3 @ w3
    dz2 = r(dh2 * (f["h2"] > 0))
    dh1 = dz2 @ w2
    dz1 = r(dh1 * (f["h1"] > 0))
    scale = 1.0 / (s * b)
    g = pack(dz1.T @ f["x"], dz2.T @ f["h1"], dz2.sum(0), dz3.T @ f["h2"], dz3.sum(0)) * scale
    glat = (dz1 @ w1[:, :LATENT]) * scale  # row i: d loss / d latent of sample i
    return loss(y, t), y, g, glat


def adam(p, m, v, g, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in float32 (as the device computes it); returns p, m, v."""
    p, m, v, g = (np.asarray(a, np.float32) for a in (p, m, v, g))
    f = np.float32
    m = f(b1) * m + (f(1) - f(b1)) * g
    v = f(b2) * v + (f(1) - f(b2)) * g * g
    c1 = f(1) - f(b1) ** f(t)
    c2 = f(1) - f(b2) ** f(t)
    p = p - f(lr) * (m / c1) / (np.sqrt(v / c2) + f(eps))
    return p, m, v
