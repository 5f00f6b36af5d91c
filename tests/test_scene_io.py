"""Scene files on the CPU: the oracle's restatement of the reference's
`.splat` and PLY readers/writers (oracle/scene_io.py) against the reference's
own tests (src/splat_format.rs:66-91, src/ply.rs:432-506), and the C ABI's
host-side rejection of malformed files (no GPU is touched: every check runs
before the upload)."""

import ctypes

import numpy as np
import pytest

from oracle import scene_io as IO
from splat_b200 import _native as N
from splat_b200.scene import Scene


def quat_rot(axis, angle):
    q = np.zeros(4, np.float32)
    q[axis] = np.sin(angle / 2)
    q[3] = np.cos(angle / 2)
    return q


def sample_scene():
    s = Scene()
    s.push([1.0, 2.0, 3.0], [0.1, 0.2, 0.3], quat_rot(1, 0.5), 0.75, [0.2, 0.4, 0.6])
    s.push([0.0, 0.0, 0.0], [0.05, 0.05, 0.05], [0, 0, 0, 1], 0.25, [1.0, 1.0, 1.0])
    s._flush()
    return s


def angle_between(a, b):
    d = abs(float(np.dot(a / np.linalg.norm(a), b / np.linalg.norm(b))))
    return 2 * np.arccos(min(d, 1.0))


def test_splat_roundtrip():
    s = Scene()
    s.push([1.0, -2.0, 3.5], [0.1, 0.2, 0.3], quat_rot(0, 0.7), 0.5, [1.0, 0.5, 0.0])
    s._flush()
    b = IO.write_splat(s)
    assert len(b) == 32
    r = IO.parse_splat(b)
    assert np.array_equal(r.positions[0], s.positions[0]) and np.array_equal(r.scales[0], s.scales[0])
    assert abs(r.opacities[0] - 0.5) < 0.01
    assert np.linalg.norm(r.colors[0] - s.colors[0]) < 0.01
    assert angle_between(r.rotations[0], s.rotations[0]) < 0.05
    with pytest.raises(ValueError):
        IO.parse_splat(bytes(33))


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian", "ascii"])
def test_ply_roundtrip(fmt):
    s = sample_scene()
    r = IO.parse_ply(IO.write_ply(s, fmt))
    assert len(r) == 2
    assert np.linalg.norm(r.positions[0] - s.positions[0]) < 1e-6
    assert np.linalg.norm(r.scales[0] - s.scales[0]) < 1e-5
    assert abs(r.opacities[0] - 0.75) < 1e-5
    assert np.linalg.norm(r.colors[0] - s.colors[0]) < 1e-5
    assert angle_between(r.rotations[0], s.rotations[0]) < 1e-3


def test_ply_roundtrip_with_sh():
    s = sample_scene()
    s.sh_degree = 1
    s.sh_rest = np.array([[i, 10 + i, 20 + i] for i in range(6)], np.float32).reshape(2, 3, 3)
    r = IO.parse_ply(IO.write_ply(s))
    assert r.sh_degree == 1
    assert np.array_equal(r.sh_rest, s.sh_rest)


def test_ply_ascii_point_cloud():
    txt = (b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\nproperty float y\nproperty float z\n"
           b"property uchar red\nproperty uchar green\nproperty uchar blue\nend_header\n0 0 0 255 0 0\n1 1 1 0 255 0\n")
    s = IO.parse_ply(txt)
    assert len(s) == 2
    assert np.array_equal(s.colors[0], [1.0, 0.0, 0.0])
    assert s.opacities[1] == 1.0


def _create(fn, data, precision=0):
    L = N.lib()
    buf = np.frombuffer(data, np.uint8) if data else np.zeros(1, np.uint8)
    h = ctypes.c_void_p()
    rc = getattr(L, fn)(buf.ctypes.data, len(data), precision, 0, ctypes.byref(h))
    return rc, L.splat_cuda_create_error().decode(), h


def test_decoders_reject_malformed_files_on_the_host(cuda_lib):
    rc, msg, h = _create("splat_cuda_create_from_splat", bytes(33))
    assert rc == N.SPLAT_ERR_INVALID_ARG and "not a multiple of 32" in msg and not h.value
    rc, msg, _ = _create("splat_cuda_create_from_ply", b"hello world")
    assert rc == N.SPLAT_ERR_INVALID_ARG and "end_header" in msg
    rc, msg, _ = _create("splat_cuda_create_from_ply", b"ply\nformat binary_little_endian 1.0\nend_header\n")
    assert rc == N.SPLAT_ERR_INVALID_ARG and "no vertex element" in msg
    full = IO.write_ply(sample_scene())
    rc, msg, _ = _create("splat_cuda_create_from_ply", full[:-10])
    assert rc == N.SPLAT_ERR_INVALID_ARG and "truncated" in msg
    rc, msg, _ = _create("splat_cuda_create_from_ply", b"nope\nend_header\n")
    assert rc == N.SPLAT_ERR_INVALID_ARG and "magic" in msg
    packed = (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\nproperty float y\n"
              b"property float z\nproperty uint packed_position\nend_header\n" + bytes(16))
    rc, msg, _ = _create("splat_cuda_create_from_ply", packed)
    assert rc == N.SPLAT_ERR_UNSUPPORTED and "packed" in msg
    nox = b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float y\nproperty float z\nend_header\n1 2\n"
    rc, msg, _ = _create("splat_cuda_create_from_ply", nox)
    assert rc == N.SPLAT_ERR_INVALID_ARG and "missing 'x'" in msg
    rc, msg, _ = _create("splat_cuda_create_from_ply", b"ply\nformat ascii 1.0\nelement vertex 2\nproperty float x\n"
                         b"property float y\nproperty float z\nend_header\n1 2 3\n")
    assert rc == N.SPLAT_ERR_INVALID_ARG and "truncated" in msg
