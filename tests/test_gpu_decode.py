"""Device-side scene decoding (splat_cuda_create_from_splat / _from_ply):
the scene the GPU decodes and finalizes from a file's bytes equals the one
splat_cuda_create uploads after the reference's reader (restated in
oracle/scene_io.py) and Scene::finalize ran on the host. Checked through the
device's own projections (bit-identical positions, depths, conics and
colours; the bbox radius k within 1e-6, since the host takes the platform's
f32 ln and the device a correctly rounded one) and exact-blend images."""

import numpy as np
import pytest

from oracle import scene_io as IO
from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer, from_ply_bytes, from_splat_bytes
from tests import scenes

pytestmark = pytest.mark.gpu


def view_of(s, yaw=0.6, pitch=0.2):
    c, r = s.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.rotate(yaw, pitch)
    return cam.view()


def compare(dev, host, s, fp16=False, w=400, h=240):
    for r in (dev, host):
        r.set_option(N.SPLAT_OPT_DEBUG_CAPTURE, 1)
        r.set_exact(True)
    v = view_of(s)
    fd, fh = Frame(), Frame()
    sd = dev.render(v, w, h, (0.1, 0.1, 0.1), fd)
    sh = host.render(v, w, h, (0.1, 0.1, 0.1), fh)
    a, b = dev.debug_dump(w, h), host.debug_dump(w, h)
    assert np.array_equal(a["visible"], b["visible"])
    vis = a["visible"]
    assert vis.sum() > 0
    exact = [0, 1, 4, 5, 6, 7]  # x, y, depth, conic
    assert np.array_equal(a["proj"][vis][:, exact], b["proj"][vis][:, exact])
    np.testing.assert_allclose(a["proj"][vis][:, 2:4], b["proj"][vis][:, 2:4], rtol=1e-6)
    assert np.array_equal(a["color"][vis], b["color"][vis])
    diff = int(np.abs(fd.pixels.astype(int) - fh.pixels.astype(int)).max())
    assert diff <= 1, diff
    assert sd.visible == sh.visible
    return int(np.sum(fd.pixels != fh.pixels))


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian"])
@pytest.mark.parametrize("degree", [0, 1, 3])
def test_ply_decode_matches_host_path(cuda_lib, fmt, degree):
    s = scenes.clusters(5000, seed=70 + degree, sh_degree=degree)
    data = IO.write_ply(s, fmt)
    host_scene = IO.parse_ply(data).finalize()
    dev = from_ply_bytes(data)
    assert dev.n == len(s)
    host = CudaRenderer(host_scene)
    compare(dev, host, host_scene)
    dev.close()
    host.close()


def test_ply_decode_types_ascii_and_defaults(cuda_lib):
    s = scenes.clusters(300, seed=80, sh_degree=1)
    # double positions, f64 opacity, int16 normals: the reader's f64 -> f32 conversions
    types = {"x": "double", "y": "double", "z": "double", "opacity": "double", "nx": "short", "ny": "short",
             "nz": "short"}
    for data in (IO.write_ply(s, "binary_little_endian", types), IO.write_ply(s, "ascii")):
        host_scene = IO.parse_ply(data).finalize()
        dev, host = from_ply_bytes(data), CudaRenderer(host_scene)
        compare(dev, host, host_scene)
        dev.close()
        host.close()
    # a coloured point cloud: u8 colours, default opacity, scale and rotation
    n = 500
    rng = np.random.default_rng(3)
    p = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    c = rng.integers(0, 256, (n, 3)).astype(np.uint8)
    txt = "ply\nformat ascii 1.0\nelement vertex %d\nproperty float x\nproperty float y\nproperty float z\n" \
          "property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n" % n
    txt += "".join(f"{float(p[i, 0])!r} {float(p[i, 1])!r} {float(p[i, 2])!r} {c[i, 0]} {c[i, 1]} {c[i, 2]}\n"
                   for i in range(n))
    data = txt.encode()
    host_scene = IO.parse_ply(data).finalize()
    dev, host = from_ply_bytes(data), CudaRenderer(host_scene)
    compare(dev, host, host_scene)
    dev.close()
    host.close()


def test_splat_decode_matches_host_path(cuda_lib):
    s = scenes.clusters(6000, seed=90, sh_degree=0)
    data = IO.write_splat(s)
    host_scene = IO.parse_splat(data).finalize()
    dev, host = from_splat_bytes(data), CudaRenderer(host_scene)
    assert dev.n == 6000
    compare(dev, host, host_scene)
    dev.close()
    host.close()


@pytest.mark.parametrize("kind", ["ply", "splat"])
def test_fp16_decode_matches_host_half_path(cuda_lib, kind):
    s = scenes.clusters(4000, seed=95, sh_degree=3 if kind == "ply" else 0)
    data = IO.write_ply(s) if kind == "ply" else IO.write_splat(s)
    host_scene = (IO.parse_ply(data) if kind == "ply" else IO.parse_splat(data)).finalize()
    loader = from_ply_bytes if kind == "ply" else from_splat_bytes
    dev = loader(data, N.SPLAT_PRECISION_FP16)
    host = CudaRenderer(host_scene.to_fp16())
    compare(dev, host, host_scene, fp16=True)
    dev.close()
    host.close()


def test_empty_files(cuda_lib):
    r = from_splat_bytes(b"")
    f = Frame()
    r.render(view_of(scenes.clusters(100, seed=1, sh_degree=0)), 64, 48, (0.2, 0.3, 0.4), f)
    assert r.n == 0 and np.all(f.pixels == f.pixels[0, 0])
    r.close()
