"""Batched rendering over the C ABI's ``splat_cuda_batch_*`` entry points:
many views of uneven resolution over several scenes, each pipeline stage one
launch over all views, recorded once as a CUDA graph and replayed.

The reference draws one view per ``Renderer::render`` call
(``src/render/mod.rs:89-96``); a batch draws every view of the list in one
replay, and each view's image is the one ``CudaRenderer.render`` draws for
it alone. Frames live in one device buffer (a torch uint8 tensor, the only
use of torch here: device memory); ``frames()`` copies them to the host.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .camera import View
from .render import CudaRenderer, RenderStats, _view_desc


@dataclass
class BatchView:
    """One view of a batch: scene index, camera, size, background, and an
    optional downsample factor (one that divides the tile shape)."""

    scene: int
    view: View
    width: int
    height: int
    background: tuple = (0.0, 0.0, 0.0)
    downsample: int = 1

    def out_size(self):
        f = max(int(self.downsample), 1)
        return self.width // f, self.height // f


class BatchRenderer:
    """A recorded batch over `scenes` (CudaRenderer handles, kept alive by the
    batch) and `views`."""

    def __init__(self, scenes: list[CudaRenderer], views: list[BatchView]):
        import torch

        L = N.lib()
        self.scenes = list(scenes)
        self.views = list(views)
        device = self.scenes[0].device
        sizes = [v.out_size() for v in self.views]
        # 256-byte aligned frames, one after another in one device buffer
        offs, o = [], 0
        for w, h in sizes:
            offs.append(o)
            o = (o + w * h * 3 + 255) // 256 * 256
        self._offsets = np.array(offs + [o], np.int64)
        total = max(o, 256)
        self.frames_dev = torch.empty(total, dtype=torch.uint8, device=f"cuda:{device}")
        base = self.frames_dev.data_ptr()
        arr = (N.BatchViewC * len(self.views))()
        for i, v in enumerate(self.views):
            c = arr[i]
            c.scene = v.scene
            c.width, c.height = v.width, v.height
            c.downsample = max(int(v.downsample), 1)
            c.view = _view_desc(v.view)
            for k in range(3):
                c.bg[k] = float(v.background[k])
            c.dev_out = base + int(self._offsets[i])
        handles = (ctypes.c_void_p * len(self.scenes))(*[s._h.value for s in self.scenes])
        b = ctypes.c_void_p()
        rc = L.splat_cuda_batch_create(handles, len(self.scenes), arr, len(self.views), ctypes.byref(b))
        if rc != N.SPLAT_OK:
            raise N.SplatError(rc, L.splat_cuda_batch_create_error().decode())
        self._b = b

    # --- configuration ------------------------------------------------------
    @property
    def config(self):
        c = N.BlendConfigC()
        N.check(N.lib().splat_cuda_batch_get_config(self._b, ctypes.byref(c)), batch=self._b)
        return (c.tile_w, c.tile_h, c.threads)

    def set_config(self, tile_w: int, tile_h: int, threads: int):
        c = N.BlendConfigC(tile_w, tile_h, threads)
        N.check(N.lib().splat_cuda_batch_set_config(self._b, ctypes.byref(c)), what="set_config", batch=self._b)

    def autotune(self, reps: int = 5):
        """Times every supported (tile shape, threads) configuration and keeps
        the fastest; returns [((tile_w, tile_h, threads), ms per batch), ...]."""
        res = (N.TuneResultC * len(N.BLEND_CONFIGS))()
        n = ctypes.c_uint32(0)
        N.check(N.lib().splat_cuda_batch_autotune(self._b, reps, res, len(res), ctypes.byref(n)), what="autotune",
                batch=self._b)
        return [((r.config.tile_w, r.config.tile_h, r.config.threads), r.ms) for r in res[: n.value]]

    def set_exact(self, exact: bool):
        N.check(N.lib().splat_cuda_batch_set_option(self._b, N.SPLAT_OPT_EXACT_BLEND, int(exact)), batch=self._b)

    def get_option(self, option: int) -> int:
        v = ctypes.c_uint64(0)
        N.check(N.lib().splat_cuda_batch_get_option(self._b, option, ctypes.byref(v)), batch=self._b)
        return int(v.value)

    def set_option(self, option: int, value: int):
        N.check(N.lib().splat_cuda_batch_set_option(self._b, option, int(value)), batch=self._b)

    def stream(self) -> int:
        return N.lib().splat_cuda_batch_get_stream(self._b) or 0

    # --- running --------------------------------------------------------------
    def run(self):
        """Launches the recorded graph (asynchronous)."""
        N.check(N.lib().splat_cuda_batch_run(self._b), what="run", batch=self._b)

    def finish(self):
        """Waits; returns (per-view RenderStats, device ms of the last batch,
        regrown). regrown: the batch overflowed its pair buffers, which have
        been grown; run it again."""
        st = (N.RenderStatsC * len(self.views))()
        ms = ctypes.c_double(0.0)
        rg = ctypes.c_int(0)
        N.check(N.lib().splat_cuda_batch_finish(self._b, st, ctypes.byref(ms), ctypes.byref(rg)), what="finish",
                batch=self._b)
        return [RenderStats.from_c(s) for s in st], ms.value, bool(rg.value)

    def render(self):
        """run + finish, again after a regrowth; returns (stats, ms)."""
        while True:
            self.run()
            stats, ms, regrown = self.finish()
            if not regrown:
                return stats, ms

    def frames(self):
        """The views' frames as host arrays (h, w, 3) uint8."""
        host = self.frames_dev.cpu().numpy()
        out = []
        for i, v in enumerate(self.views):
            w, h = v.out_size()
            o = int(self._offsets[i])
            out.append(host[o: o + w * h * 3].reshape(h, w, 3).copy())
        return out

    def close(self):
        if getattr(self, "_b", None):
            N.lib().splat_cuda_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
