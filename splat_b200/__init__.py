"""splat_b200 — a B200 (sm_100a) backend for farmerchris/splat's Gaussian-splat
tile rasterizer, behind the reference's ``Renderer`` interface.

The compute path is ``libsplat_cuda.so`` (hand-written CUDA kernels, C ABI in
``include/splat_cuda.h``); this package is the host-side mirror of the
reference's renderer API (``src/render/mod.rs``), camera (``src/camera.rs``)
and scene (``src/scene.rs``) over that ABI.
"""

from .camera import MAX_PITCH, OrbitCamera, UpAxis, View, to_radians
from .render import (ALPHA_MAX, ALPHA_MIN, DILATION, MAX_DIM, T_MIN, TILE, Backend, CudaRenderer, Frame,
                     RenderStats, Renderer, create)
from .scene import SH_C0, HalfScene, Scene, coeffs_for_degree, covariance, degree_from_rest_count

__all__ = [
    "MAX_PITCH", "OrbitCamera", "UpAxis", "View", "to_radians", "ALPHA_MAX", "ALPHA_MIN", "DILATION", "MAX_DIM",
    "T_MIN", "TILE", "Backend", "CudaRenderer", "Frame", "RenderStats", "Renderer", "create", "SH_C0", "HalfScene", "Scene",
    "coeffs_for_degree", "covariance", "degree_from_rest_count",
]
