"""FP16 scene storage (scales, rotations, opacities, base colour and SH as
IEEE binary16; positions f32) with FP32 projection and blending, and FP64
only for 2D covariances whose f32 determinant falls below 1e-6.

Gates:
* every splat not on the FP64 path projects bit-identically to the oracle's
  f32 `project` run on the decoded values (the device forms the covariance
  from the halves with the reference's Scene::finalize + covariance order);
* exact-blend images equal the oracle `cpu` backend on the decoded scene;
* splats on the FP64 path: their count equals the oracle's count of f32
  determinants below 1e-6, and their conics agree with a double-precision
  computation to 1e-4 relative;
* per-image error against the FP64 naive rasterizer is stated (PSNR, max
  abs) and bounded: >= 45 dB on the decoded values, >= 40 dB against the
  FP64 rendering of the original f32 parameters (storage error included).
"""

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis, View
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu

FP64_BELOW = np.float32(1e-6)


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _views(s, n=3):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    out = [cam.view()]
    for i in range(n - 1):
        cam.rotate(1.3, 0.2 * (-1) ** i)
        cam.zoom(0.55 if i % 2 == 0 else 1.6)
        out.append(cam.view())
    return out


def _frame(r, view, w, h, bg=(0.0, 0.0, 0.0), exact=False):
    r.set_exact(exact)
    f = Frame()
    st = r.render(view, w, h, bg, f)
    return f.pixels.copy(), st


def _max_abs(a, b):
    return int(np.max(np.abs(a.astype(int) - b.astype(int)))) if a.size else 0


@pytest.mark.parametrize("degree,size", [(3, (640, 360)), (1, (97, 53)), (0, (320, 180))])
def test_fp16_projection_bit_exact_on_decoded_values(oracle, degree, size):
    s = scenes.clusters(20_000, seed=17 + degree, sh_degree=degree)
    half = s.to_fp16()
    dec = half.decoded_scene()
    w, h = size
    r = CudaRenderer(half)
    assert r.precision == N.SPLAT_PRECISION_FP16
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.set_option(N.SPLAT_OPT_BBOX_PAIRS, 1)  # the reference's pairs: every tile of the pixel bbox
    for view in _views(s):
        r.render(view, w, h, (0.1, 0.2, 0.3), Frame())
        d = r.debug_dump(w, h)
        ref, vis = oracle.project(dec, view, w, h)
        det = oracle.project_det(dec, view, w, h)
        f32_path = det >= FP64_BELOW  # +inf: culled before the determinant
        assert r.fp64_conics() == int(np.sum(~f32_path & (det != np.inf)))
        m = vis & f32_path
        assert np.array_equal(d["visible"][f32_path], vis[f32_path]), "culling differs"
        p, o = d["proj"][m], ref[m]
        for di, oi in [(0, 0), (1, 1), (2, 10), (3, 11), (4, 9), (5, 2), (6, 3), (7, 4)]:
            assert np.array_equal(p[:, di].view(np.uint32), o[:, oi].view(np.uint32)), f"field {di} differs"
        assert np.array_equal(d["color"][m].view(np.uint32), o[:, 5:8].view(np.uint32)), "colour differs"
        # Keys and ranges stay bit-exact against the CPU recomputation.
        pr = d["proj"]
        keys, vals, ranges = oracle.bin_sort(pr[:, 0], pr[:, 1], pr[:, 2], pr[:, 3], pr[:, 4], d["visible"], w, h)
        assert np.array_equal(d["keys"], keys) and np.array_equal(d["values"], vals)
        assert np.array_equal(d["ranges"], ranges)
    r.close()


def test_fp16_exact_images_equal_cpu_on_decoded_scene(oracle):
    s = scenes.clusters(20_000, seed=23, sh_degree=3)
    half = s.to_fp16()
    dec = half.decoded_scene()
    r = CudaRenderer(half)
    cpu = oracle.CpuTiled(dec)
    for view in _views(s):
        want, _ = cpu.render(view, 480, 270, (0.1, 0.2, 0.3))
        got, _ = _frame(r, view, 480, 270, (0.1, 0.2, 0.3), exact=True)
        if r.fp64_conics() == 0:
            assert np.array_equal(got, want), f"{np.sum(got != want)} channels differ"
        fast, _ = _frame(r, view, 480, 270, (0.1, 0.2, 0.3))
        assert oracle.psnr(fast, want) >= 60.0 and _max_abs(fast, want) <= 2
    cpu.close()
    r.close()


def _conics_f64(dec, view, w, h, oracle):
    """2D conics in double precision from the decoded values (the same
    formulas as project(), src/render/mod.rs:199-272, all in f64)."""
    ctx = oracle.project_ctx(view, w, h).astype(np.float64)
    rot = ctx[0:9].reshape(3, 3)
    eye = ctx[9:12]
    focal, near, lim_x, lim_y = ctx[12], ctx[17], ctx[18], ctx[19]
    p = dec.positions.astype(np.float64)
    t = (p - eye) @ rot.T
    tz = t[:, 2]
    with np.errstate(all="ignore"):
        inv_z = 1.0 / tz
        jx = np.clip(t[:, 0] * inv_z, -lim_x, lim_x)
        jy = np.clip(t[:, 1] * inv_z, -lim_y, lim_y)
        f = focal * inv_z
        j0 = np.stack([f, np.zeros_like(f), -f * jx], 1)
        j1 = np.stack([np.zeros_like(f), f, -f * jy], 1)
        t0 = j0 @ rot
        t1 = j1 @ rot
        q = dec.rotations.astype(np.float64)
        q = q / np.linalg.norm(q, axis=1, keepdims=True)
        x, y, z, ww = q.T
        R = np.stack([
            np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - ww * z), 2 * (x * z + ww * y)], 1),
            np.stack([2 * (x * y + ww * z), 1 - 2 * (x * x + z * z), 2 * (y * z - ww * x)], 1),
            np.stack([2 * (x * z - ww * y), 2 * (y * z + ww * x), 1 - 2 * (x * x + y * y)], 1)], 1)
        M = R * dec.scales.astype(np.float64)[:, None, :]
        S = M @ np.transpose(M, (0, 2, 1))
        s0 = np.einsum("nij,nj->ni", S, t0)
        s1 = np.einsum("nij,nj->ni", S, t1)
        a = np.sum(t0 * s0, 1) + 0.3
        b = np.sum(t1 * s0, 1)
        c = np.sum(t1 * s1, 1) + 0.3
        det = a * c - b * b
        return np.stack([c / det, -b / det, a / det], 1), tz > near


def test_fp64_conics_for_near_singular_covariances(oracle):
    s = scenes.needles(20_000)
    half = s.to_fp16()
    dec = half.decoded_scene()
    view = View.looking_along_z(np.zeros(3, np.float32))
    w, h = 640, 360
    r = CudaRenderer(half)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.render(view, w, h, (0.0, 0.0, 0.0), Frame())
    d = r.debug_dump(w, h)
    det = oracle.project_det(dec, view, w, h)
    low = det < FP64_BELOW
    n64 = r.fp64_conics()
    print(f"needles: {n64} of {len(s)} splats took the FP64 conic path")
    assert n64 == int(np.sum(low)) and n64 > 0
    want, _ = _conics_f64(dec, view, w, h, oracle)
    m = low & d["visible"]
    assert np.sum(m) > 0
    got = d["proj"][m][:, 5:8].astype(np.float64)
    ref = want[m]
    scale = np.max(np.abs(ref), axis=1, keepdims=True)
    assert np.max(np.abs(got - ref) / scale) < 1e-4
    # The f32 splats keep the oracle's f32 values bit for bit.
    ref32, vis32 = oracle.project(dec, view, w, h)
    k = ~low & vis32
    assert np.array_equal(d["visible"][~low], vis32[~low])
    assert np.array_equal(d["proj"][k][:, 5:8].view(np.uint32), ref32[k][:, 2:5].view(np.uint32))
    r.close()


def test_fp32_scenes_never_take_the_fp64_path():
    s = scenes.needles(4_000)
    r = CudaRenderer(s)
    r.render(View.looking_along_z(np.zeros(3, np.float32)), 320, 180, (0.0, 0.0, 0.0), Frame())
    assert r.fp64_conics() == 0
    r.close()


@pytest.mark.parametrize("degree", [3, 0])
def test_fp16_error_against_fp64_naive(oracle, degree):
    s = scenes.clusters(30_000, seed=31 + degree, sh_degree=degree)
    half = s.to_fp16()
    r = CudaRenderer(half)
    dec = half.decoded()
    orig = {"positions": s.positions, "scales": s.scales, "rotations": s.rotations, "opacities": s.opacities,
            "colors": s.colors, "sh_rest": s.sh_rest, "sh_degree": s.sh_degree}
    w, h = 640, 360
    for i, view in enumerate(_views(s)):
        got, _ = _frame(r, view, w, h)
        ref64, _, _ = oracle.render_naive_f64(dec, view, w, h)
        src64, _, _ = oracle.render_naive_f64(orig, view, w, h)
        p, e = oracle.psnr(got, ref64), _max_abs(got, ref64)
        ps, es = oracle.psnr(got, src64), _max_abs(got, src64)
        print(f"deg {degree} frame {i}: vs FP64 naive (decoded) {p:.2f} dB max {e}; "
              f"(f32 source) {ps:.2f} dB max {es}; fp64 conics {r.fp64_conics()}")
        assert p >= 45.0, (p, e)
        assert ps >= 40.0, (ps, es)
    r.close()
