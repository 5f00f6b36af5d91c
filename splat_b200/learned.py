"""Learned colour: a 16-latent-per-splat MLP that replaces degree-3 SH.

No counterpart in the reference, whose splats carry 48 SH floats
(``src/scene.rs:20-23``) evaluated by ``sh::eval_rest`` (``src/sh.rs:39-64``).
Here each splat keeps 16 fp16 latents and one shared MLP decodes
(latent, view direction) -> RGB on the tensor cores, inside the projection
kernel. ``Learner`` trains the latents and the MLP on the device from an
SH scene's exact colours; ``learned_renderer`` builds a renderer from the
trained values and the FP16 geometry.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .render import CudaRenderer
from .scene import HalfScene


@dataclass
class LearnConfig:
    directions: int = 256   # Fibonacci-sphere directions per splat
    batch: int = 65536      # samples per step (multiple of 128)
    lr: float = 1e-3
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    seed: int = 0

    def to_c(self) -> N.LearnConfigC:
        return N.LearnConfigC(self.directions, self.batch, self.lr, self.beta1, self.beta2, self.eps,
                              self.seed & ((1 << 64) - 1))


@dataclass
class LearnStats:
    steps: int
    epochs: float
    mean_loss: float
    last_loss: float
    ms: float
    steps_per_epoch: int
    samples_per_epoch: int


def _ptr(a):
    return None if a is None else a.ctypes.data


class Learner:
    """Trains latents + MLP on `sh_renderer`'s scene (its device, its exact SH)."""

    def __init__(self, sh_renderer: CudaRenderer, config: LearnConfig = LearnConfig()):
        L = N.lib()
        h = ctypes.c_void_p()
        rc = L.splat_cuda_learner_create(sh_renderer._h, ctypes.byref(config.to_c()), ctypes.byref(h))
        if rc != N.SPLAT_OK:
            raise N.SplatError(rc, L.splat_cuda_learner_create_error().decode())
        self._h = h
        self._scene = sh_renderer  # must outlive the learner
        self.n = sh_renderer.n
        self.config = config

    def _check(self, rc, what):
        if rc != N.SPLAT_OK:
            raise N.SplatError(rc, f"{what}: {N.lib().splat_cuda_learner_last_error(self._h).decode()}")

    def option(self, opt: int) -> int:
        v = ctypes.c_uint64(0)
        self._check(N.lib().splat_cuda_learner_get_option(self._h, opt, ctypes.byref(v)), "get_option")
        return int(v.value)

    def set_option(self, opt: int, value: int):
        self._check(N.lib().splat_cuda_learner_set_option(self._h, opt, int(value)), "set_option")

    @property
    def steps_per_epoch(self) -> int:
        return self.option(N.LEARN_STEPS_PER_EPOCH)

    def train(self, steps: int) -> LearnStats:
        st = N.LearnStatsC()
        self._check(N.lib().splat_cuda_learner_train(self._h, int(steps), ctypes.byref(st)), "train")
        return LearnStats(int(st.steps), st.epochs, st.mean_loss, st.last_loss, st.ms, int(st.steps_per_epoch),
                          int(st.samples_per_epoch))

    def train_epochs(self, epochs: float) -> LearnStats:
        return self.train(int(round(epochs * self.steps_per_epoch)))

    def params(self):
        """fp32 masters: (params (7248,), latents (n, 16))."""
        p = np.zeros(N.MLP_PARAMS, np.float32)
        lat = np.zeros((self.n, N.MLP_LATENT), np.float32)
        self._check(N.lib().splat_cuda_learner_params(self._h, _ptr(p), _ptr(lat), None, None), "params")
        return p, lat

    def params_f16(self):
        """The fp16 values the kernels use (bit patterns): (params, latents (n, 16))."""
        p = np.zeros(N.MLP_PARAMS, np.uint16)
        lat = np.zeros((self.n, N.MLP_LATENT), np.uint16)
        self._check(N.lib().splat_cuda_learner_params(self._h, None, None, _ptr(p), _ptr(lat)), "params")
        return p, lat

    def set_params(self, params=None, latents=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        lat = None if latents is None else np.ascontiguousarray(latents, np.float32).reshape(self.n, N.MLP_LATENT)
        self._check(N.lib().splat_cuda_learner_set_params(self._h, _ptr(p), _ptr(lat)), "set_params")

    def save_state(self) -> bytes:
        """The training state (parameters, latents, Adam moments, step count)
        as bytes; `load_state` on a learner of the same scene and
        configuration resumes from it."""
        n = N.lib().splat_cuda_learner_state_bytes(self._h)
        buf = ctypes.create_string_buffer(n)
        self._check(N.lib().splat_cuda_learner_save_state(self._h, buf, n), "save_state")
        return buf.raw

    def load_state(self, state: bytes):
        buf = ctypes.create_string_buffer(bytes(state), len(state))
        self._check(N.lib().splat_cuda_learner_load_state(self._h, buf, len(state)), "load_state")

    def save(self, path: str):
        with open(path, "wb") as f:
            f.write(self.save_state())

    def load(self, path: str):
        with open(path, "rb") as f:
            self.load_state(f.read())

    def step_debug(self):
        """One step; returns its gradient (d params, d latents (n, 16))."""
        g = np.zeros(N.MLP_PARAMS, np.float32)
        gl = np.zeros((self.n, N.MLP_LATENT), np.float32)
        self._check(N.lib().splat_cuda_learner_step_debug(self._h, _ptr(g), _ptr(gl)), "step_debug")
        return g, gl

    def directions(self) -> np.ndarray:
        d = np.zeros((self.config.directions, 3), np.float32)
        self._check(N.lib().splat_cuda_learner_directions(self._h, _ptr(d)), "directions")
        return d

    def close(self):
        if getattr(self, "_h", None):
            N.lib().splat_cuda_learner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def learned_renderer(geometry: HalfScene, latents_f16: np.ndarray, params_f16: np.ndarray,
                     device: int = 0) -> CudaRenderer:
    """A renderer over FP16 geometry whose colours come from the MLP."""
    L = N.lib()
    n = len(geometry)
    keep = [np.ascontiguousarray(geometry.positions, np.float32), geometry.scales, geometry.rotations,
            geometry.opacities]
    d = N.SceneDesc()
    d.n = n
    d.sh_degree = 0
    d.precision = N.SPLAT_PRECISION_FP16
    d.positions, d.scales_f16, d.rotations_f16, d.opacities_f16 = [a.ctypes.data for a in keep]
    lat = np.ascontiguousarray(latents_f16, np.uint16).reshape(n, N.MLP_LATENT)
    prm = np.ascontiguousarray(params_f16, np.uint16).reshape(N.MLP_PARAMS)
    h = ctypes.c_void_p()
    rc = L.splat_cuda_create_learned(ctypes.byref(d), lat.ctypes.data, prm.ctypes.data, device, ctypes.byref(h))
    if rc != N.SPLAT_OK:
        raise N.SplatError(rc, L.splat_cuda_create_error().decode())
    r = CudaRenderer.__new__(CudaRenderer)
    r._keep = None
    r._h = h
    r.n = n
    r.device = device
    r.precision = N.SPLAT_PRECISION_FP16
    return r


def mlp_gradient(params, latents_f16, dirs, targets, device: int = 0):
    """The training kernel on explicit samples: (loss, outputs (B, 3),
    d params (7248,), d latents (B, 16)) of the mean squared error."""
    p = np.ascontiguousarray(params, np.float32)
    lat = np.ascontiguousarray(latents_f16, np.uint16)
    d = np.ascontiguousarray(dirs, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    b = len(lat)
    g = np.zeros(N.MLP_PARAMS, np.float32)
    gl = np.zeros((b, N.MLP_LATENT), np.float32)
    y = np.zeros((b, 3), np.float32)
    loss = ctypes.c_double(0)
    rc = N.lib().splat_cuda_mlp_gradient(device, p.ctypes.data, lat.ctypes.data, d.ctypes.data, t.ctypes.data, b,
                                         g.ctypes.data, gl.ctypes.data, y.ctypes.data, ctypes.byref(loss))
    if rc != N.SPLAT_OK:
        raise N.SplatError(rc, "mlp_gradient")
    return loss.value, y, g, gl
