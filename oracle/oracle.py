"""ORACLE — test infrastructure only.

ctypes wrapper of ``oracle/_build/libsplat_oracle.so``, the C++ restatement of
farmerchris/splat's CPU rasterizers (``src/render/{mod,cpu,naive,radix,simd}.rs``,
``src/sh.rs``, ``src/scene.rs``, ``src/term.rs``, ``src/bench.rs``). Only the
tests, the smoke check and bench.py's CPU-baseline leg import this module, as
the checker; the product library never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libsplat_oracle.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_project.argtypes = [ctypes.c_uint64, ctypes.c_uint32] + [_f32p] * 6 + [
            ctypes.c_uint32, ctypes.c_uint32, _f32p, _u8p]
        L.oracle_project_det.argtypes = [ctypes.c_uint64, ctypes.c_uint32] + [_f32p] * 6 + [
            ctypes.c_uint32, ctypes.c_uint32, _f32p]
        L.oracle_project_ctx.argtypes = [_f32p, ctypes.c_uint32, ctypes.c_uint32, _f32p]
        L.oracle_eval_rest.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p]
        L.oracle_covariance.argtypes = [_f32p, _f32p, _f32p]
        L.oracle_exp_neg.argtypes = [_f32p, _f32p, ctypes.c_uint64]
        L.oracle_sort_hi32.argtypes = [_u64p, ctypes.c_uint64]
        L.oracle_fix_ties.argtypes = [_u64p, ctypes.c_uint64, _u32p]
        L.oracle_spread3.argtypes = [ctypes.c_uint32]
        L.oracle_spread3.restype = ctypes.c_uint32
        L.oracle_bounds.argtypes = [ctypes.c_uint64, _f32p, _f32p]
        L.oracle_downsample.argtypes = [_u8p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u8p]
        L.oracle_psnr.argtypes = [_u8p, _u8p, ctypes.c_uint64]
        L.oracle_psnr.restype = ctypes.c_double
        L.oracle_render_naive.argtypes = [ctypes.c_uint64, ctypes.c_uint32] + [_f32p] * 6 + [
            ctypes.c_uint32, ctypes.c_uint32, _f32p, _u8p, _f64p]
        L.oracle_render_naive_f64.argtypes = [ctypes.c_uint64, ctypes.c_uint32] + [_f32p] * 7 + [
            ctypes.c_uint32, ctypes.c_uint32, _f32p, _u8p, _f64p, _f64p]
        L.oracle_cpu_create.argtypes = [ctypes.c_uint64, ctypes.c_uint32] + [_f32p] * 5 + [ctypes.c_uint32]
        L.oracle_cpu_create.restype = ctypes.c_void_p
        L.oracle_cpu_render.argtypes = [ctypes.c_void_p, _f32p, ctypes.c_uint32, ctypes.c_uint32, _f32p, _u8p, _f64p]
        L.oracle_cpu_threads.argtypes = [ctypes.c_void_p]
        L.oracle_cpu_threads.restype = ctypes.c_uint32
        L.oracle_cpu_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_bin_sort.argtypes = [ctypes.c_uint64] + [_f32p] * 5 + [_u8p] + [ctypes.c_uint32] * 4 + [
            _u64p, _u32p, ctypes.c_uint64, _u32p]
        L.oracle_bin_sort.restype = ctypes.c_int64
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _scene_ptrs(scene):
    pos = _f32(scene.positions)
    op = _f32(scene.opacities)
    col = _f32(scene.colors)
    cov = _f32(scene.cov3d)
    rest = _f32(scene.sh_rest if scene.sh_degree > 0 else np.zeros(1, np.float32))
    keep = (pos, op, col, cov, rest)
    return keep, [_p(a, _f32p) for a in keep]


def _view(view) -> np.ndarray:
    return _f32(view.to_array())


def _stats(s):
    return {"visible": int(s[0]), "overlaps": int(s[1]), "project_ms": s[2], "sort_ms": s[3],
            "raster_ms": s[4], "total_ms": s[5]}


def project(scene, view, w, h):
    """Per-splat project(): returns (out[n,12], visible[n] bool)."""
    n = len(scene.opacities)
    keep, ptrs = _scene_ptrs(scene)
    out = np.zeros((n, 12), np.float32)
    vis = np.zeros(n, np.uint8)
    v = _view(view)
    lib().oracle_project(n, scene.sh_degree, *ptrs, _p(v, _f32p), w, h, _p(out, _f32p), _p(vis, _u8p))
    return out, vis.astype(bool)


def project_det(scene, view, w, h):
    """The f32 2D covariance determinant project() computes per splat (+inf
    where the splat is culled before it)."""
    n = len(scene.opacities)
    keep, ptrs = _scene_ptrs(scene)
    det = np.zeros(n, np.float32)
    lib().oracle_project_det(n, scene.sh_degree, *ptrs, _p(_view(view), _f32p), w, h, _p(det, _f32p))
    return det


def project_ctx(view, w, h):
    v = _view(view)
    out = np.zeros(20, np.float32)
    lib().oracle_project_ctx(_p(v, _f32p), w, h, _p(out, _f32p))
    return out


def eval_rest(degree, rest, direction):
    rest = _f32(rest)
    d = _f32(direction)
    out = np.zeros(3, np.float32)
    lib().oracle_eval_rest(degree, _p(rest, _f32p), _p(d, _f32p), _p(out, _f32p))
    return out


def covariance(scale, quat_xyzw):
    s = _f32(scale)
    q = _f32(quat_xyzw)
    out = np.zeros(6, np.float32)
    lib().oracle_covariance(_p(s, _f32p), _p(q, _f32p), _p(out, _f32p))
    return out


def exp_neg(x):
    x = _f32(x).ravel()
    out = np.zeros_like(x)
    lib().oracle_exp_neg(_p(x, _f32p), _p(out, _f32p), x.size)
    return out


def sort_hi32(keys):
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    lib().oracle_sort_hi32(_p(k, _u64p), k.size)
    return k


def fix_ties(keys, orig):
    k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
    o = np.ascontiguousarray(orig, dtype=np.uint32)
    lib().oracle_fix_ties(_p(k, _u64p), k.size, _p(o, _u32p))
    return k


def spread3(v):
    return lib().oracle_spread3(v)


def bounds(positions):
    pos = _f32(positions)
    out = np.zeros(4, np.float32)
    lib().oracle_bounds(len(pos), _p(pos, _f32p), _p(out, _f32p))
    return out[:3].copy(), float(out[3])


def downsample(img, factor):
    """term::downsample on an (h, w, 3) u8 image."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    f = max(factor, 1)
    out = np.zeros((h // f, w // f, 3), np.uint8)
    lib().oracle_downsample(_p(img, _u8p), w, h, factor, _p(out, _u8p))
    return out


def psnr(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    if a.shape != b.shape:
        return 0.0
    return lib().oracle_psnr(_p(a, _u8p), _p(b, _u8p), a.size // 3)


def render_naive(scene, view, w, h, bg=(0.0, 0.0, 0.0)):
    """CpuNaive::render (FP32): returns (image (h, w, 3) u8, stats)."""
    n = len(scene.opacities)
    keep, ptrs = _scene_ptrs(scene)
    img = np.zeros((h, w, 3), np.uint8)
    st = np.zeros(6, np.float64)
    v = _view(view)
    b = _f32(bg)
    rc = lib().oracle_render_naive(n, scene.sh_degree, *ptrs, _p(v, _f32p), w, h, _p(b, _f32p), _p(img, _u8p),
                                   _p(st, _f64p))
    if rc:
        raise ValueError(f"frame {w}x{h} exceeds the 16384 pixel limit")
    return img, _stats(st)


def render_naive_f64(decoded, view, w, h, bg=(0.0, 0.0, 0.0)):
    """FP64 naive rasterizer on decoded FP16 parameters (dict of float32 arrays:
    positions, scales, rotations (x,y,z,w), opacities, colors, sh_rest, sh_degree).
    Returns (image u8, linear float64 image, stats)."""
    n = len(decoded["opacities"])
    arrs = [_f32(decoded[k]) for k in ("positions", "scales", "rotations", "opacities", "colors")]
    deg = int(decoded["sh_degree"])
    rest = _f32(decoded["sh_rest"] if deg > 0 else np.zeros(1, np.float32))
    img = np.zeros((h, w, 3), np.uint8)
    lin = np.zeros((h, w, 3), np.float64)
    st = np.zeros(6, np.float64)
    v = _view(view)
    b = _f32(bg)
    rc = lib().oracle_render_naive_f64(n, deg, *[_p(a, _f32p) for a in arrs], _p(rest, _f32p), _p(v, _f32p), w, h,
                                       _p(b, _f32p), _p(img, _u8p), _p(lin, _f64p), _p(st, _f64p))
    if rc:
        raise ValueError(f"frame {w}x{h} exceeds the 16384 pixel limit")
    return img, lin, _stats(st)


class CpuTiled:
    """CpuTiled (the reference's default `cpu` backend), restated."""

    def __init__(self, scene, threads: int = 0):
        self._keep, ptrs = _scene_ptrs(scene)
        self._h = lib().oracle_cpu_create(len(scene.opacities), scene.sh_degree, *ptrs, threads)
        self.threads = lib().oracle_cpu_threads(self._h)

    def name(self):
        return "cpu"

    def render(self, view, w, h, bg=(0.0, 0.0, 0.0), out=None):
        img = out if out is not None else np.zeros((h, w, 3), np.uint8)
        st = np.zeros(6, np.float64)
        v = _view(view)
        b = _f32(bg)
        rc = lib().oracle_cpu_render(self._h, _p(v, _f32p), w, h, _p(b, _f32p), _p(img, _u8p), _p(st, _f64p))
        if rc:
            raise ValueError(f"frame {w}x{h} exceeds the 16384 pixel limit")
        return img, _stats(st)

    def close(self):
        if self._h:
            lib().oracle_cpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bin_sort(x, y, ext_x, ext_y, depth, visible, w, h, cap=None, tile=(16, 16)):
    """CPU recomputation of sorted (tile<<32 | depth bits) keys, splat values and
    per-tile [begin, end) ranges from projected values (tile_w x tile_h tiles)."""
    n = len(x)
    arrs = [_f32(a) for a in (x, y, ext_x, ext_y, depth)]
    vis = np.ascontiguousarray(visible, dtype=np.uint8)
    tw, th = tile
    tiles = ((w + tw - 1) // tw) * ((h + th - 1) // th)
    if cap is None:
        cap = max(16, int(np.sum(vis)) * 64)
    while True:
        keys = np.zeros(cap, np.uint64)
        vals = np.zeros(cap, np.uint32)
        ranges = np.zeros(2 * tiles, np.uint32)
        p = lib().oracle_bin_sort(n, *[_p(a, _f32p) for a in arrs], _p(vis, _u8p), w, h, tw, th, _p(keys, _u64p),
                                  _p(vals, _u32p), cap, _p(ranges, _u32p))
        if p >= 0:
            return keys[:p], vals[:p], ranges.reshape(tiles, 2)
        cap *= 4
