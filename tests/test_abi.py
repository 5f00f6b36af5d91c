"""The C ABI library loads and exports every function include/*.h declares
(CPU only: no compute calls), and the host-side mirror behaves like the
reference's types."""

import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, Scene, UpAxis, View, covariance, synth
from splat_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(splat_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(cuda_lib):
    names = declared_functions()
    assert names, "no declarations found"
    assert set(N.EXPORTS) <= names
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    missing = names - exported
    assert not missing, f"declared but not exported: {missing}"
    for n in names:
        getattr(cuda_lib, n)
    assert cuda_lib.splat_cuda_abi_version() == 1
    assert cuda_lib.splat_cuda_backend_name() == b"cuda"


def test_abi_struct_layouts():
    # splat_scene_desc: u64 + 2 u32 + 9 pointers; view: 14 floats; stats: 2 u64 + 4 f64.
    assert ctypes.sizeof(N.SceneDesc) == 8 + 8 + 9 * 8
    assert ctypes.sizeof(N.ViewDesc) == 14 * 4
    assert ctypes.sizeof(N.RenderStatsC) == 48


def test_null_arguments_are_rejected_without_a_gpu(cuda_lib):
    h = ctypes.c_void_p()
    assert cuda_lib.splat_cuda_create(None, 0, ctypes.byref(h)) == N.SPLAT_ERR_INVALID_ARG
    assert cuda_lib.splat_cuda_create(None, 0, None) == N.SPLAT_ERR_INVALID_ARG
    assert cuda_lib.splat_cuda_render(None, None, 1, 1, None, 1, None, 0, None) == N.SPLAT_ERR_INVALID_ARG
    assert cuda_lib.splat_cuda_destroy(None) == N.SPLAT_OK
    assert cuda_lib.splat_cuda_last_error(None) == b""
    d = N.SceneDesc()
    d.n = 1
    d.sh_degree = 4
    assert cuda_lib.splat_cuda_create(ctypes.byref(d), 0, ctypes.byref(h)) == N.SPLAT_ERR_INVALID_ARG
    assert b"sh_degree" in cuda_lib.splat_cuda_create_error()


def test_frame_resize_and_pixel_limit():
    f = Frame()
    f.resize(16384, 1)
    assert f.pixels.shape == (1, 16384, 3)
    with pytest.raises(ValueError, match="pixel limit"):
        Frame().resize(65536, 65537)


def test_camera_basis_orthonormal_right_handed():
    # src/camera.rs:203-218
    for up in UpAxis:
        c = OrbitCamera.new(np.zeros(3, np.float32), 1.0, up)
        c.rotate(0.7, 0.3)
        v = c.view()
        for a in (v.right, v.down):
            assert abs(np.linalg.norm(a) - 1) < 1e-5
        assert abs(np.dot(v.right, v.down)) < 1e-5
        assert np.linalg.norm(np.cross(v.right, v.down) - v.forward) < 1e-5
        assert np.dot(-v.down, up.vector()) > 0


def test_camera_target_projects_to_center_and_pitch_clamps():
    # src/camera.rs:220-236
    c = OrbitCamera.new(np.zeros(3, np.float32), 1.0, UpAxis.NEG_Y)
    p = c.view().to_camera(c.target)
    assert abs(p[0]) < 1e-5 and abs(p[1]) < 1e-5 and abs(p[2] - c.distance) < 1e-4
    c.rotate(0.0, 10.0)
    assert c.pitch <= np.float32(89 * np.pi / 180) + 1e-6
    c.rotate(0.0, -20.0)
    assert c.pitch >= -np.float32(89 * np.pi / 180) - 1e-6
    d = c.distance
    c.rotate(1.0, 0.5)
    c.zoom(0.5)
    c.pan(0.3, 0.1)
    c.reset()
    assert c.distance == d and np.all(c.target == 0)
    assert UpAxis.parse("-y") == UpAxis.NEG_Y and UpAxis.parse("Z") == UpAxis.POS_Z
    with pytest.raises(ValueError):
        UpAxis.parse("w")


def test_scene_covariance_matches_oracle(oracle):
    s = synth.cluster_scene(2000, seed=5, sh_degree=1)
    for i in range(0, 2000, 97):
        want = oracle.covariance(s.scales[i], s.rotations[i])
        assert np.array_equal(s.cov3d[i].view(np.uint32), want.view(np.uint32))


def test_scene_finalize_and_bounds(oracle):
    s = Scene()
    s.positions = np.zeros((1, 3), np.float32)
    with pytest.raises(ValueError):
        s.finalize()
    t = Scene()
    for i in range(100):
        t.push((i / 100, 0, 0), (1, 1, 1), (0, 0, 0, 1), 1.0, (1, 1, 1))
    t.push((1e6, 1e6, 1e6), (1, 1, 1), (0, 0, 0, 1), 1.0, (1, 1, 1))
    t.finalize()
    c, r = t.bounds()
    assert r < 1.0 and abs(c[0] - 0.5) < 0.05
    oc, orr = oracle.bounds(t.positions)
    assert np.allclose(c, oc) and abs(r - orr) < 1e-6


def test_synthetic_scenes_are_seeded():
    a = synth.cluster_scene(1000, seed=1)
    b = synth.cluster_scene(1000, seed=1)
    c = synth.cluster_scene(1000, seed=2)
    assert np.array_equal(a.positions, b.positions) and np.array_equal(a.sh_rest, b.sh_rest)
    assert not np.array_equal(a.positions, c.positions)
    assert len(synth.lattice_scene()) == 14 ** 3
    # SplitMix64 known value: the first output for seed 0 (gen.rs:28-34).
    assert int(synth.splitmix_u64(0, 1)[0]) == 0xE220A8397B1DCDAF


def test_scene_precision_validation_without_a_gpu(cuda_lib):
    h = ctypes.c_void_p()
    d = N.SceneDesc()
    d.n = 1
    d.precision = 7
    assert cuda_lib.splat_cuda_create(ctypes.byref(d), 0, ctypes.byref(h)) == N.SPLAT_ERR_UNSUPPORTED
    d.precision = N.SPLAT_PRECISION_FP16
    assert cuda_lib.splat_cuda_create(ctypes.byref(d), 0, ctypes.byref(h)) == N.SPLAT_ERR_INVALID_ARG
    assert b"FP16" in cuda_lib.splat_cuda_create_error()


def test_half_scene_round_trip():
    from splat_b200 import HalfScene  # noqa: F401
    from tests import scenes

    s = scenes.clusters(2_000, seed=3, sh_degree=2)
    half = s.to_fp16()
    assert half.sh.shape == (2_000, 9, 3) and half.sh.dtype == np.uint16
    # 12 B position + 2 * (3 + 4 + 1 + 27) B of halves per degree-2 splat
    assert half.positions.nbytes + half.scales.nbytes + half.rotations.nbytes + half.opacities.nbytes + \
        half.sh.nbytes == 2_000 * (12 + 2 * (3 + 4 + 1 + 27))
    d = half.decoded()
    for k, tol in [("scales", 2 ** -11), ("opacities", 2 ** -11), ("colors", 2 ** -11), ("sh_rest", 2 ** -11)]:
        a = np.asarray(getattr(s, k), np.float32).reshape(d[k].shape)
        assert np.all(np.abs(d[k] - a) <= tol * np.maximum(np.abs(a), 2 ** -14)), k
    assert np.array_equal(d["positions"], s.positions)
    ds = half.decoded_scene()
    scale = np.max(np.abs(s.cov3d[:, [0, 3, 5]]), axis=1, keepdims=True)  # largest variance per splat
    assert np.all(np.abs(ds.cov3d - s.cov3d) <= 5e-3 * scale)


def test_batch_abi_layouts_and_validation_without_a_gpu(cuda_lib):
    # splat_batch_view: 4 u32 + view (14 f32) + 3 f32 + u32 + pointer.
    assert ctypes.sizeof(N.BatchViewC) == 16 + 56 + 12 + 4 + 8
    assert ctypes.sizeof(N.BlendConfigC) == 12
    assert ctypes.sizeof(N.TuneResultC) == 24
    b = ctypes.c_void_p()
    assert cuda_lib.splat_cuda_batch_create(None, 0, None, 0, ctypes.byref(b)) == N.SPLAT_ERR_INVALID_ARG
    assert b"no scenes" in cuda_lib.splat_cuda_batch_create_error()
    handles = (ctypes.c_void_p * 1)(None)
    views = (N.BatchViewC * 1)()
    assert cuda_lib.splat_cuda_batch_create(handles, 1, views, 1, ctypes.byref(b)) == N.SPLAT_ERR_INVALID_ARG
    assert b"null scene" in cuda_lib.splat_cuda_batch_create_error()
    assert cuda_lib.splat_cuda_batch_destroy(None) == N.SPLAT_OK
    assert cuda_lib.splat_cuda_batch_run(None) == N.SPLAT_ERR_INVALID_ARG
    assert cuda_lib.splat_cuda_batch_last_error(None) == b""
    assert len(N.BLEND_CONFIGS) == 9 and len(set(N.BLEND_CONFIGS)) == 9


def test_c_driver_builds_against_the_header(cuda_lib, tmp_path):
    """include/splat_cuda.h is valid C99 and the library links from C."""
    from tests import c_driver

    assert os.path.exists(c_driver.build(str(tmp_path)))
