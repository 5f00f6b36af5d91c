"""The renderer interface of farmerchris/splat (``src/render/mod.rs``) over the
sm_100a backend's C ABI.

``Renderer``, ``Frame``, ``RenderStats``, ``Backend`` and ``create`` keep the
reference's names, argument meaning and error behaviour: ``render`` resizes
the caller's frame and fills it (``mod.rs:86-97``); frames above
``MAX_DIM`` are rejected with the reference's "pixel limit" message
(``mod.rs:35-41``); a zero-sized frame returns default stats
(``cpu.rs:120-122``); backend creation fails with an error, not a crash
(``mod.rs:115-134``).
"""

from __future__ import annotations

import ctypes
import enum
from abc import ABC, abstractmethod
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .camera import View
from .scene import HalfScene, Scene

# src/render/mod.rs:23-33
DILATION = np.float32(0.3)
ALPHA_MIN = np.float32(1.0 / 255.0)
ALPHA_MAX = np.float32(0.99)
T_MIN = np.float32(1e-4)
MAX_DIM = 16384
TILE = 16  # src/render/cpu.rs:34


def _pixel_count(width: int, height: int) -> int:
    if width > MAX_DIM or height > MAX_DIM:
        raise ValueError(f"frame {width}x{height} exceeds the {MAX_DIM} pixel limit")
    return width * height


class Frame:
    """8-bit RGB image, row-major (``mod.rs:43-70``); ``pixels`` is (h, w, 3) u8."""

    def __init__(self, width: int = 0, height: int = 0):
        _pixel_count(width, height)
        self.width = width
        self.height = height
        self.pixels = np.zeros((height, width, 3), np.uint8)

    def resize(self, width: int, height: int):
        _pixel_count(width, height)
        self.width, self.height = width, height
        if self.pixels.shape != (height, width, 3):
            self.pixels = np.zeros((height, width, 3), np.uint8)

    def get(self, x: int, y: int):
        return self.pixels[y, x].tolist()


@dataclass
class RenderStats:
    """``RenderStats`` (``mod.rs:72-83``); ``overlaps`` = (splat, tile) pairs."""

    visible: int = 0
    overlaps: int = 0
    project_ms: float = 0.0
    sort_ms: float = 0.0
    raster_ms: float = 0.0
    total_ms: float = 0.0

    @staticmethod
    def from_c(s: N.RenderStatsC) -> "RenderStats":
        return RenderStats(int(s.visible), int(s.overlaps), s.project_ms, s.sort_ms, s.raster_ms, s.total_ms)


class Renderer(ABC):
    """A rasterizer backend bound to one scene (``mod.rs:85-97``)."""

    @abstractmethod
    def name(self) -> str: ...

    @abstractmethod
    def render(self, view: View, width: int, height: int, background, frame: Frame) -> RenderStats: ...


class Backend(enum.Enum):
    """Backends of this package. The reference's ``cpu``/``cpu-naive``/``gpu``
    backends are its own Rust/wgpu code and are not part of this package."""

    CUDA = "cuda"

    @staticmethod
    def all():
        return [Backend.CUDA]


def _view_desc(view: View) -> N.ViewDesc:
    v = N.ViewDesc()
    a = view.to_array()
    for i in range(3):
        v.eye[i], v.right[i], v.down[i], v.forward[i] = a[i], a[3 + i], a[6 + i], a[9 + i]
    v.fov_y, v.near_plane = a[12], a[13]
    return v


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class CudaRenderer(Renderer):
    """The sm_100a backend: uploads the scene once, renders views on `device`."""

    def __init__(self, scene, device: int = 0):
        """`scene`: a finalized Scene (FP32 storage) or a HalfScene (FP16
        storage of scales, rotations, opacities and SH)."""
        L = N.lib()
        n = len(scene)
        d = N.SceneDesc()
        d.n = n
        d.sh_degree = scene.sh_degree
        if isinstance(scene, HalfScene):
            self._keep = [_f32(scene.positions), scene.scales, scene.rotations, scene.opacities, scene.sh]
            d.precision = N.SPLAT_PRECISION_FP16
            d.positions, d.scales_f16, d.rotations_f16, d.opacities_f16, d.sh_f16 = [
                a.ctypes.data for a in self._keep]
        else:
            self._keep = [_f32(scene.positions), _f32(scene.opacities), _f32(scene.colors), _f32(scene.cov3d),
                          _f32(scene.sh_rest.reshape(n, -1) if scene.sh_degree > 0 else np.zeros(1, np.float32))]
            d.precision = N.SPLAT_PRECISION_FP32
            d.positions, d.opacities, d.colors, d.cov3d, d.sh_rest = [a.ctypes.data for a in self._keep]
        self.precision = d.precision
        h = ctypes.c_void_p()
        rc = L.splat_cuda_create(ctypes.byref(d), device, ctypes.byref(h))
        if rc != N.SPLAT_OK:
            raise N.SplatError(rc, L.splat_cuda_create_error().decode())
        self._keep = None  # the scene lives on the device now
        self._h = h
        self.n = n
        self.device = device

    # --- Renderer ---------------------------------------------------------
    def name(self) -> str:
        return N.lib().splat_cuda_backend_name().decode()

    def render(self, view: View, width: int, height: int, background=(0.0, 0.0, 0.0), frame: Frame = None,
               downsample: int = 1) -> RenderStats:
        """Render into `frame` (resized to the output size). With
        downsample f > 1 the frame is term::downsample'd by f on the device
        and `frame` becomes floor(w/f) x floor(h/f)."""
        f = max(int(downsample), 1)
        if frame is None:
            frame = Frame()
        _pixel_count(width, height)
        frame.resize(width // f, height // f)
        bg = _f32(background)
        st = N.RenderStatsC()
        rc = N.lib().splat_cuda_render(self._h, ctypes.byref(_view_desc(view)), width, height,
                                       bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), f,
                                       frame.pixels.ctypes.data, frame.pixels.nbytes, ctypes.byref(st))
        N.check(rc, self._h, "render")
        return RenderStats.from_c(st)

    def render_cells(self, view: View, width: int, height: int, background=(0.0, 0.0, 0.0), downsample: int = 1,
                     mode: int = N.SPLAT_CELLS_TRUECOLOR, stats: bool = False):
        """The terminal widget's cells (``HalfBlockImage``, ``term.rs:109-130``)
        of the downsampled frame, computed on the device: a (rows, cols, 6)
        array of fg RGB + bg RGB (truecolor) or (rows, cols, 2) of xterm-256
        indices (ansi256)."""
        f = max(int(downsample), 1)
        _pixel_count(width, height)
        cols, rows = width // f, (height // f) // 2
        per = 6 if mode == N.SPLAT_CELLS_TRUECOLOR else 2
        out = np.zeros((rows, cols, per), np.uint8)
        c, r = ctypes.c_uint32(0), ctypes.c_uint32(0)
        st = N.RenderStatsC()
        bg = _f32(background)
        rc = N.lib().splat_cuda_render_cells(self._h, ctypes.byref(_view_desc(view)), width, height,
                                             bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), f, mode,
                                             out.ctypes.data if out.size else None, out.nbytes, ctypes.byref(c),
                                             ctypes.byref(r), ctypes.byref(st))
        N.check(rc, self._h, "render_cells")
        return (out, RenderStats.from_c(st)) if stats else out

    def render_rows(self, view: View, width: int, height: int, background, row0: int, rows: int,
                    out: np.ndarray = None, stats: bool = False):
        """Rows [row0, row0 + rows) of the width x height frame, bit for bit
        as `render` draws them (splat_cuda_render_rows): only the tile rows
        of the window are binned, sorted and blended. Returns a (rows, width,
        3) u8 array (`out` if given, C-contiguous)."""
        _pixel_count(width, height)
        if out is None:
            out = np.empty((rows, width, 3), np.uint8)
        if out.shape != (rows, width, 3) or out.dtype != np.uint8 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous (rows, width, 3) uint8 array")
        bg = _f32(background)
        st = N.RenderStatsC()
        rc = N.lib().splat_cuda_render_rows(self._h, ctypes.byref(_view_desc(view)), width, height,
                                            bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), row0, rows,
                                            out.ctypes.data_as(ctypes.c_void_p), out.nbytes, ctypes.byref(st))
        N.check(rc, self._h, "render_rows")
        return (out, RenderStats.from_c(st)) if stats else out

    # --- splat-sharded frames ---------------------------------------------------
    def shard_records(self, view: View, width: int, height: int, row_bounds, send=None):
        """The record exchange's sender side (splat_cuda_shard_records): this
        renderer's scene is one shard of the splats; its splats are projected
        for the whole frame and each visible one goes, as a
        SPLAT_RECORD_BYTES-byte record, to every row window [row_bounds[k],
        row_bounds[k + 1]) its pixel bbox meets. Returns (records, counts,
        visible): a uint8 CUDA tensor of sum(counts) records, window after
        window, each window's in scene order (`send`, a uint8 CUDA tensor, is
        used when large enough), the records per window and the shard's
        visible splats."""
        import torch

        _pixel_count(width, height)
        bounds = np.ascontiguousarray(row_bounds, np.uint32)
        nw = len(bounds) - 1
        counts = np.zeros(max(nw, 1), np.uint64)
        vis = ctypes.c_uint64(0)
        rb = N.SPLAT_RECORD_BYTES
        if send is None:
            send = torch.empty(max(self.n, 1) * rb + 16, dtype=torch.uint8, device=f"cuda:{self.device}")
        for _ in range(2):
            base = send.data_ptr()
            off = (-base) % 16  # the records start 16-byte aligned
            cap = max(send.numel() - off, 0) // rb
            rc = N.lib().splat_cuda_shard_records(
                self._h, ctypes.byref(_view_desc(view)), width, height, nw,
                bounds.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), base + off if cap else None, cap,
                counts.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(vis))
            if rc == N.SPLAT_ERR_CAPACITY:
                send = torch.empty(int(counts[:nw].sum()) * rb + 16, dtype=torch.uint8, device=send.device)
                continue
            N.check(rc, self._h, "shard_records")
            total = int(counts[:nw].sum())
            return send[off:off + total * rb], [int(c) for c in counts[:nw]], int(vis.value)
        raise N.SplatError(N.SPLAT_ERR_CAPACITY, "shard_records: the send buffer did not grow")

    def render_records(self, view: View, width: int, height: int, background, records, row0: int, rows: int,
                       out=None, stats: bool = False):
        """Rows [row0, row0 + rows) of the frame drawn from received records
        (splat_cuda_render_records): `records` is a uint8 CUDA tensor of
        whole records on this renderer's device (the senders' runs for this
        window, concatenated in shard order). `out`: a (rows, width, 3)
        uint8 numpy array (host) or CUDA tensor (written in place); a new
        numpy array when None."""
        import torch

        _pixel_count(width, height)
        rb = N.SPLAT_RECORD_BYTES
        if records.numel() % rb:
            raise ValueError("records must hold whole records of SPLAT_RECORD_BYTES bytes")
        n = records.numel() // rb
        if n and records.data_ptr() % 16:
            records = records.clone()  # the records must start 16-byte aligned
        if out is None:
            out = np.empty((rows, width, 3), np.uint8)
        if isinstance(out, torch.Tensor):
            if tuple(out.shape) != (rows, width, 3) or out.dtype != torch.uint8 or not out.is_contiguous():
                raise ValueError("out must be a contiguous (rows, width, 3) uint8 tensor")
            if out.is_cuda and out.device.index != self.device:
                raise ValueError(f"out is on {out.device}, the renderer on cuda:{self.device}")
            ptr, nbytes = out.data_ptr(), out.numel()
        else:
            if out.shape != (rows, width, 3) or out.dtype != np.uint8 or not out.flags["C_CONTIGUOUS"]:
                raise ValueError("out must be a C-contiguous (rows, width, 3) uint8 array")
            ptr, nbytes = out.ctypes.data, out.nbytes
        bg = _f32(background)
        st = N.RenderStatsC()
        rc = N.lib().splat_cuda_render_records(self._h, ctypes.byref(_view_desc(view)), width, height,
                                               bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                               records.data_ptr() if n else None, n, row0, rows, ptr, nbytes,
                                               ctypes.byref(st))
        N.check(rc, self._h, "render_records")
        return (out, RenderStats.from_c(st)) if stats else out

    # --- device-side entry points --------------------------------------------
    def render_into(self, view: View, width: int, height: int, background, out_ptr: int, out_bytes: int,
                    downsample: int = 1) -> RenderStats:
        """Render into caller-owned HOST memory at `out_ptr` (e.g. a pinned
        torch tensor's data_ptr()); blocks until the frame is there."""
        bg = _f32(background)
        st = N.RenderStatsC()
        rc = N.lib().splat_cuda_render(self._h, ctypes.byref(_view_desc(view)), width, height,
                                       bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), max(int(downsample), 1),
                                       out_ptr, out_bytes, ctypes.byref(st))
        N.check(rc, self._h, "render")
        return RenderStats.from_c(st)

    def render_device(self, view: View, width: int, height: int, background, dev_ptr: int, out_bytes: int,
                      downsample: int = 1):
        """Enqueue a frame into DEVICE memory `dev_ptr` on this renderer's
        stream; no host synchronisation (pair with `finish`)."""
        bg = _f32(background)
        rc = N.lib().splat_cuda_render_device(self._h, ctypes.byref(_view_desc(view)), width, height,
                                              bg.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                              max(int(downsample), 1), dev_ptr, out_bytes)
        N.check(rc, self._h, "render_device")

    def finish(self):
        """Wait for enqueued frames; returns (stats of the last, regrown)."""
        st = N.RenderStatsC()
        regrown = ctypes.c_int(0)
        N.check(N.lib().splat_cuda_finish(self._h, ctypes.byref(st), ctypes.byref(regrown)), self._h, "finish")
        return RenderStats.from_c(st), bool(regrown.value)

    def set_stream(self, stream_ptr: int):
        N.check(N.lib().splat_cuda_set_stream(self._h, stream_ptr or None), self._h, "set_stream")

    def stream(self) -> int:
        return N.lib().splat_cuda_get_stream(self._h) or 0

    def set_option(self, option: int, value: int):
        N.check(N.lib().splat_cuda_set_option(self._h, option, int(value)), self._h, "set_option")

    def get_option(self, option: int) -> int:
        v = ctypes.c_uint64(0)
        N.check(N.lib().splat_cuda_get_option(self._h, option, ctypes.byref(v)), self._h, "get_option")
        return int(v.value)

    def set_blend_config(self, tile_w: int, tile_h: int, threads: int):
        """Tile shape and blend threads: (8, 8), (16, 16) or (32, 16) tiles with
        128, 256 or 512 threads. The image does not depend on it."""
        self.set_option(N.SPLAT_OPT_BLEND_CONFIG, N.pack_blend_config(tile_w, tile_h, threads))

    def set_exact(self, exact: bool):
        """Blend with the reference cpu backend's exact f32 arithmetic."""
        self.set_option(N.SPLAT_OPT_EXACT_BLEND, int(exact))

    def fp64_conics(self) -> int:
        """Splats of the last completed frame whose 2D covariance was inverted
        in FP64 (FP16 scenes: determinant below 1e-6 in FP32)."""
        return self.get_option(N.SPLAT_OPT_FP64_CONICS)

    def debug_dump(self, width: int, height: int):
        """Intermediate buffers of the last frame (needs SPLAT_OPT_DEBUG_CAPTURE):
        dict with proj (n, 8), visible (n,), color (n, 3), keys, values, ranges."""
        L = N.lib()
        n = self.n
        proj = np.zeros((n, 8), np.float32)
        vis = np.zeros(n, np.uint8)
        col = np.zeros((n, 3), np.float32)
        npairs = ctypes.c_uint64(0)
        packed = self.get_option(N.SPLAT_OPT_BLEND_CONFIG)
        tw, th = packed & 0xFF, (packed >> 8) & 0xFF
        tiles = ((width + tw - 1) // tw) * ((height + th - 1) // th)
        ranges = np.zeros((tiles, 2), np.uint32)
        N.check(L.splat_cuda_debug_dump(self._h, None, None, None, None, None, 0, None, 0, ctypes.byref(npairs)),
                self._h, "debug_dump")
        p = int(npairs.value)
        keys = np.zeros(max(p, 1), np.uint64)
        vals = np.zeros(max(p, 1), np.uint32)
        N.check(L.splat_cuda_debug_dump(self._h, proj.ctypes.data, vis.ctypes.data, col.ctypes.data,
                                        keys.ctypes.data, vals.ctypes.data, p, ranges.ctypes.data, ranges.size,
                                        ctypes.byref(npairs)), self._h, "debug_dump")
        return {"proj": proj, "visible": vis.astype(bool), "color": col, "keys": keys[:p], "values": vals[:p],
                "ranges": ranges}

    def close(self):
        if getattr(self, "_h", None):
            N.lib().splat_cuda_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _from_handle(h, n: int, precision: int, device: int) -> CudaRenderer:
    r = CudaRenderer.__new__(CudaRenderer)
    r._keep = None
    r._h = h
    r.n = n
    r.device = device
    r.precision = precision
    return r


def _load_bytes(fn, data: bytes, precision: int, device: int) -> CudaRenderer:
    L = N.lib()
    buf = np.frombuffer(data, np.uint8) if len(data) else np.zeros(1, np.uint8)
    h = ctypes.c_void_p()
    rc = getattr(L, fn)(buf.ctypes.data, len(data), precision, device, ctypes.byref(h))
    if rc != N.SPLAT_OK:
        raise N.SplatError(rc, L.splat_cuda_create_error().decode())
    r = _from_handle(h, 0, precision, device)
    r.n = r.get_option(N.SPLAT_OPT_SCENE_SPLATS)
    return r


def from_splat_bytes(data: bytes, precision: int = N.SPLAT_PRECISION_FP32, device: int = 0) -> CudaRenderer:
    """A renderer for the bytes of a ``.splat`` file, decoded and finalized on
    the device (``splat_format::parse`` + ``Scene::finalize``)."""
    return _load_bytes("splat_cuda_create_from_splat", data, precision, device)


def from_ply_bytes(data: bytes, precision: int = N.SPLAT_PRECISION_FP32, device: int = 0) -> CudaRenderer:
    """A renderer for the bytes of a 3DGS PLY file, decoded and finalized on
    the device (``ply::parse`` + ``Scene::finalize``)."""
    return _load_bytes("splat_cuda_create_from_ply", data, precision, device)


def load(path: str, precision: int = N.SPLAT_PRECISION_FP32, device: int = 0) -> CudaRenderer:
    """``Scene::load`` (``src/scene.rs:96-110``) straight to a device scene:
    the format is chosen by extension (``.ply`` or ``.splat``)."""
    with open(path, "rb") as fh:
        data = fh.read()
    base = path.replace("\\", "/").rsplit("/", 1)[-1]
    ext = base.rsplit(".", 1)[-1].lower() if "." in base else ""
    if ext == "splat":
        return from_splat_bytes(data, precision, device)
    if ext == "ply" or data.startswith(b"ply"):
        return from_ply_bytes(data, precision, device)
    raise ValueError(f"unknown file type (expected .ply or .splat): {path}")


def create(backend: Backend, scene: Scene, device: int = 0) -> Renderer:
    """``render::create`` (``mod.rs:115-121``)."""
    if backend == Backend.CUDA:
        return CudaRenderer(scene, device)
    raise ValueError(f"unknown backend {backend!r}")
