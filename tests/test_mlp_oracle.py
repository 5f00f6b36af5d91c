"""CPU checks of the learned-colour oracle (oracle/mlp_oracle.py): its SH
targets against the C++ restatement of sh::eval_rest, its backward pass
against finite differences of its forward pass, its shuffle's bijectivity,
its Fibonacci directions and its Adam step. These pin the checker the GPU
tests compare the tensor-core kernels against."""

import numpy as np
import pytest

from oracle import mlp_oracle as M


def random_params(rng, scale=1.0):
    w1 = np.zeros((64, 32))
    w1[:, :20] = rng.normal(0, 0.4, (64, 20)) * scale
    w2 = rng.normal(0, 0.2, (64, 64)) * scale
    b2 = rng.normal(0, 0.1, 64) * scale
    w3 = np.zeros((16, 64))
    w3[:3] = rng.normal(0, 0.2, (3, 64)) * scale
    b3 = np.zeros(16)
    b3[:3] = rng.normal(0, 0.1, 3)
    return M.pack(w1, w2, b2, w3, b3)


def unit(rng, n):
    d = rng.normal(size=(n, 3))
    return d / np.linalg.norm(d, axis=1, keepdims=True)


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_eval_rest_matches_cpp_restatement(oracle, degree):
    rng = np.random.default_rng(degree)
    per = (degree + 1) ** 2 - 1
    rest = rng.normal(0, 0.3, (50, per, 3)).astype(np.float32)
    d = unit(rng, 50).astype(np.float32)
    got = M.eval_rest(degree, rest, d)
    want = np.stack([oracle.eval_rest(degree, rest[i], d[i]) for i in range(50)])
    np.testing.assert_allclose(got, want, atol=2e-6)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    b = 6
    p = random_params(rng)
    lat = rng.normal(0, 0.5, (b, 16))
    d = unit(rng, b)
    t = rng.uniform(0, 1, (b, 3))
    _, _, g, glat = M.backward(p, lat, d, t, emulate=False)

    def f(pp, ll):
        return M.loss(M.forward(pp, ll, d, emulate=False)["y"], t)

    h = 1e-6
    # every parameter that can carry a gradient (a sample)
    idx = np.concatenate([rng.choice(np.arange(0, 20), 6) + 32 * rng.integers(0, 64, 6),
                          M.W2 + rng.integers(0, 4096, 12), M.B2 + rng.integers(0, 64, 6),
                          M.W3 + rng.integers(0, 192, 8), M.B3 + np.arange(3)])
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        num = (f(p + e, lat) - f(p - e, lat)) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])
    for s in range(b):
        for k in range(0, 16, 3):
            e = np.zeros_like(lat)
            e[s, k] = h
            num = (f(p, lat + e) - f(p, lat - e)) / (2 * h)
            assert abs(num - glat[s, k]) <= 1e-6 + 1e-4 * abs(num)
    # inputs 20-31 and output rows 3-15 carry no gradient
    assert np.all(g[M.W1:M.W2].reshape(64, 32)[:, 20:] == 0)
    assert np.all(g[M.W3:M.B3].reshape(16, 64)[3:] == 0) and np.all(g[M.B3 + 3:] == 0)


@pytest.mark.parametrize("m", [1, 2, 777, 4096, 131_072, 300 * 64])
def test_shuffle_is_a_bijection(m):
    bits = max(1, int(np.ceil(np.log2(m)))) if m > 1 else 1
    for key in (M.epoch_key(0, 0), M.epoch_key(5, 3)):
        p = M.shuffle_index(np.arange(m, dtype=np.uint64), m, key, bits)
        assert np.array_equal(np.sort(p), np.arange(m, dtype=np.uint64))


def test_step_samples_cover_an_epoch_once():
    n, dirs, batch = 37, 16, 128
    spe = (n * dirs + batch - 1) // batch
    seen = np.concatenate([M.step_samples(k, n, dirs, batch, 9)[0] * dirs + M.step_samples(k, n, dirs, batch, 9)[1]
                           for k in range(spe)])
    assert len(seen) == n * dirs
    assert np.array_equal(np.sort(seen), np.arange(n * dirs))
    # the next epoch is a different order
    nxt = M.step_samples(spe, n, dirs, batch, 9)
    assert not np.array_equal(nxt[0] * dirs + nxt[1], seen[:batch])


def test_fibonacci_directions():
    d = M.fibonacci_dirs(256)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    assert abs(d[:, 1].mean()) < 1e-6  # symmetric in y
    assert d[0, 1] == np.float32(1.0 - 1.0 / 256)


def test_adam_first_step_is_lr_times_sign():
    g = np.array([1e-3, -2.0, 0.5], np.float32)
    p, m, v = M.adam(np.zeros(3), np.zeros(3), np.zeros(3), g, 1)
    np.testing.assert_allclose(p, -1e-3 * np.sign(g), rtol=1e-4)
    assert m.dtype == np.float32 and v.dtype == np.float32


def test_targets_clamped():
    rng = np.random.default_rng(1)
    rest = rng.normal(0, 2.0, (100, 15, 3))
    col = rng.normal(0.5, 1.0, (100, 3))
    t = M.sh_targets(col, rest, 3, unit(rng, 100))
    assert t.min() >= 0.0 and t.max() <= 1.0 and (t == 0).any() and (t == 1).any()
