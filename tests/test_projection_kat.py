"""Closed-form known answers for the EWA projection (src/render/mod.rs:201-272).

For a view at the origin looking along +z (rotation = identity) and a splat
at t = (X, Y, Z) with 3D covariance diag(sx^2, sy^2, sz^2), the projection is

  x = f X / Z + cx,   y = f Y / Z + cy,   depth = Z
  J = f / Z [[1, 0, -u], [0, 1, -v]],  u = clamp(X / Z), v = clamp(Y / Z)
  (a, b, c) = J Sigma J^T + 0.3 I
            = (f/Z)^2 (sx^2 + u^2 sz^2,  u v sz^2,  sy^2 + v^2 sz^2) + (0.3, 0, 0.3)
  conic = (c, -b, a) / (a c - b^2)
  ext = k (sqrt a, sqrt c),  k = sqrt(2 ln(255 opacity))

evaluated here in float64. The oracle (the C++ restatement of `project`)
must agree to f32 rounding: it is then pinned to the reference's formula in
absolute terms, not only through relative tests; the device projection
must agree the same way (and equals the oracle bit for bit elsewhere).
Culling known answers: opacity below 1/255, depth at or behind the near
plane and splats entirely off screen produce nothing.
"""

import numpy as np
import pytest

from splat_b200 import View
from splat_b200.scene import Scene

f32 = np.float32
W, H, FOV = 640, 480, 0.9


def view():
    return View(np.zeros(3, f32), np.array([1, 0, 0], f32), np.array([0, 1, 0], f32), np.array([0, 0, 1], f32),
                f32(FOV), f32(0.05))


# (position, scales, opacity, colour)
CASES = [
    ((0.0, 0.0, 4.0), (0.05, 0.05, 0.05), 0.9, (0.2, 0.5, 0.8)),    # isotropic, on the axis
    ((0.0, 0.0, 10.0), (0.3, 0.1, 0.02), 0.5, (1.0, 0.0, 0.0)),     # anisotropic, on the axis
    ((0.7, -0.4, 3.0), (0.04, 0.04, 0.04), 0.99, (0.0, 1.0, 0.0)),  # isotropic, off the axis
    ((-1.1, 0.6, 5.0), (0.02, 0.08, 0.3), 0.2, (0.5, 0.5, 0.5)),    # anisotropic, off the axis (sz enters a, b, c)
    ((3.0, 0.0, 2.0), (0.5, 0.5, 0.5), 0.9, (1.0, 1.0, 1.0)),       # X/Z beyond the Jacobian clamp, bbox on screen
]
CULLED = [
    ((0.0, 0.0, 4.0), (0.05, 0.05, 0.05), 0.003, (1, 1, 1)),        # opacity < 1/255
    ((0.0, 0.0, 0.04), (0.05, 0.05, 0.05), 0.9, (1, 1, 1)),         # in front of the near plane
    ((0.0, 0.0, -3.0), (0.05, 0.05, 0.05), 0.9, (1, 1, 1)),         # behind the camera
    ((40.0, 0.0, 4.0), (0.05, 0.05, 0.05), 0.9, (1, 1, 1)),         # off screen to the right
]


def scene(cases):
    s = Scene()
    for p, sc, op, c in cases:
        s.push(p, sc, (0, 0, 0, 1), op, c)
    return s.finalize()


def closed_form(p, sc, op):
    X, Y, Z = (float(f32(v)) for v in p)
    f = (H * 0.5) / np.tan(FOV * 0.5)
    lim_x, lim_y = 1.3 * (W * 0.5 / f), 1.3 * (H * 0.5 / f)
    u = min(max(X / Z, -lim_x), lim_x)
    v = min(max(Y / Z, -lim_y), lim_y)
    g = (f / Z) ** 2
    sx2, sy2, sz2 = (float(f32(s)) ** 2 for s in sc)
    a = g * (sx2 + u * u * sz2) + 0.3
    b = g * (u * v * sz2)
    c = g * (sy2 + v * v * sz2) + 0.3
    det = a * c - b * b
    k = np.sqrt(2.0 * np.log(float(f32(op)) * 255.0))
    return dict(x=f * X / Z + W * 0.5, y=f * Y / Z + H * 0.5, depth=Z, conic=(c / det, -b / det, a / det),
                ext=(k * np.sqrt(a), k * np.sqrt(c)))


def check(out, vis, colors):
    # out: x, y, conic a, b, c, colour r, g, b, opacity, depth, ext_x, ext_y
    assert vis.all()
    for i, (p, sc, op, col) in enumerate(CASES):
        want = closed_form(p, sc, op)
        o = out[i]
        np.testing.assert_allclose(o[0], want["x"], rtol=2e-6, atol=1e-4)
        np.testing.assert_allclose(o[1], want["y"], rtol=2e-6, atol=1e-4)
        np.testing.assert_allclose(o[9], want["depth"], rtol=1e-7)
        np.testing.assert_allclose(o[2:5], want["conic"], rtol=2e-5, atol=1e-9)
        np.testing.assert_allclose(o[10:12], want["ext"], rtol=2e-5)
        np.testing.assert_allclose(colors[i], col, rtol=1e-6)
    # On the axis: x, y are the principal point exactly and the conic is diagonal.
    for i in (0, 1):
        assert out[i, 0] == f32(W * 0.5) and out[i, 1] == f32(H * 0.5) and out[i, 3] == 0.0


def test_oracle_projection_closed_form(oracle):
    out, vis = oracle.project(scene(CASES), view(), W, H)
    check(out, vis, out[:, 5:8])
    _, vis = oracle.project(scene(CULLED), view(), W, H)
    assert not vis.any()


@pytest.mark.gpu
def test_device_projection_closed_form(oracle, cuda_lib):
    from splat_b200 import Frame
    from splat_b200 import _native as N
    from splat_b200.render import CudaRenderer

    s = scene(CASES)
    r = CudaRenderer(s)
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    r.render(view(), W, H, (0, 0, 0), Frame())
    d = r.debug_dump(W, H)
    r.close()
    p = d["proj"]  # x, y, ext_x, ext_y, depth, conic a, b, c
    out = np.zeros((len(CASES), 12), np.float32)
    out[:, 0], out[:, 1], out[:, 10], out[:, 11], out[:, 9] = p[:, 0], p[:, 1], p[:, 2], p[:, 3], p[:, 4]
    out[:, 2:5] = p[:, 5:8]
    check(out, d["visible"], d["color"])
    r = CudaRenderer(scene(CULLED))
    r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
    st = r.render(view(), W, H, (0, 0, 0), Frame())
    assert st.visible == 0 and not r.debug_dump(W, H)["visible"].any()
    r.close()
