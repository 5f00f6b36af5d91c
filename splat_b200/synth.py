"""Seeded synthetic scenes for the benchmark and test workloads.

The random source is the reference's SplitMix64 (``src/gen.rs:21-54``):
uniform f32 = (u64 >> 40) / 2^24, standard normals by Box–Muller with
u clamped at 1e-7, evaluated in binary32. Draw k of a stream seeded with s
is mix(s + (k + 1) * 0x9E3779B97F4A7C15), so a stream vectorises. Every
attribute of a scene draws from its own stream, seeded from the scene seed
and the attribute's index, so attributes are independent of one another.

Workloads (no public dataset is involved; these stand in for captures):

* ``lattice_scene``   — 14^3 isotropic splats on [-1, 1]^3, scale 0.03
  (stored as a log-scale and activated with exp), identity rotation,
  opacity 0.9, SH degree 0, colour = lattice index / 13.
* ``cluster_scene``   — N anisotropic splats from 64 isotropic clusters
  (centres U[-5, 5]^3, sigma 0.6); log-scales N(-4, 0.6) per axis; uniform
  random unit quaternions (normalised 4 x N(0, 1)); opacity logits N(0, 1.5)
  through a sigmoid; SH DC N(0, 0.5) -> base colour SH_C0 * dc + 0.5; the
  higher SH coefficients N(0, 0.08). Activations follow ``src/ply.rs:276-316``.
"""

from __future__ import annotations

import numpy as np

from .camera import OrbitCamera, UpAxis, to_radians
from .scene import SH_C0, Scene

f32 = np.float32
GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
SEED_MIX = 0x632BE59BD9B4E019
MASK64 = (1 << 64) - 1


def splitmix_u64(seed: int, count: int, offset: int = 0) -> np.ndarray:
    """Draws offset .. offset+count-1 of SplitMix64 seeded with `seed`."""
    k = np.arange(offset + 1, offset + count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & MASK64) + k * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
    return z ^ (z >> np.uint64(31))


def uniform(seed: int, count: int) -> np.ndarray:
    """``Rng::f``: uniform in [0, 1) as f32."""
    return (splitmix_u64(seed, count) >> np.uint64(40)).astype(np.float32) / f32(1 << 24)


def normal(seed: int, count: int) -> np.ndarray:
    """``Rng::normal`` (Box–Muller), consuming two draws per value."""
    u = uniform(seed, 2 * count).reshape(count, 2)
    a = np.maximum(u[:, 0], f32(1e-7))
    v = u[:, 1]
    return (np.sqrt(f32(-2.0) * np.log(a)) * np.cos(f32(2.0 * np.pi) * v)).astype(np.float32)


def stream_seed(seed: int, attr: int) -> int:
    """Seed of attribute `attr`'s stream: the first SplitMix64 output of
    seed ^ ((attr + 1) * SEED_MIX)."""
    s = (seed ^ (((attr + 1) * SEED_MIX) & MASK64)) & MASK64
    return int(splitmix_u64(s, 1)[0])


def lattice_scene(n_side: int = 14, scale: float = 0.03, opacity: float = 0.9) -> Scene:
    idx = np.arange(n_side, dtype=np.float32)
    i, j, k = np.meshgrid(idx, idx, idx, indexing="ij")
    t = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1) / f32(n_side - 1)
    s = Scene()
    s.positions = (t * f32(2.0) - f32(1.0)).astype(np.float32)
    n = len(s.positions)
    log_scale = np.full((n, 3), np.log(f32(scale)), np.float32)
    s.scales = np.exp(log_scale).astype(np.float32)
    s.rotations = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
    s.opacities = np.full(n, opacity, np.float32)
    s.colors = t.astype(np.float32)
    s.sh_degree = 0
    return s.finalize()


def cluster_scene(n: int = 1_200_000, seed: int = 0x5EED0001, sh_degree: int = 3, clusters: int = 64,
                  sh_code_dim: int = 0) -> Scene:
    """sh_code_dim = k > 0: the higher SH coefficients are not independent
    but generated from a k-dimensional code per splat, rest = B z with z ~
    N(0, I_k) and B a fixed (seeded) basis scaled so that each coefficient
    still has standard deviation 0.08 - a scene whose view-dependent colour
    carries k numbers per splat (as correlated SH of captured scenes does)
    instead of 45."""
    s = Scene()
    cl = (splitmix_u64(stream_seed(seed, 0), n) % np.uint64(clusters)).astype(np.int64)
    centres = (f32(-5.0) + f32(10.0) * uniform(stream_seed(seed, 1), clusters * 3)).reshape(clusters, 3)
    off = (f32(0.6) * normal(stream_seed(seed, 2), 3 * n)).reshape(n, 3)
    s.positions = (centres[cl] + off).astype(np.float32)
    log_scale = (f32(-4.0) + f32(0.6) * normal(stream_seed(seed, 3), 3 * n)).reshape(n, 3)
    s.scales = np.exp(log_scale).astype(np.float32)
    q = normal(stream_seed(seed, 4), 4 * n).reshape(n, 4)
    s.rotations = q  # normalised by finalize
    logit = f32(1.5) * normal(stream_seed(seed, 5), n)
    s.opacities = (f32(1.0) / (f32(1.0) + np.exp(-logit))).astype(np.float32)
    dc = (f32(0.5) * normal(stream_seed(seed, 6), 3 * n)).reshape(n, 3)
    s.colors = (dc * SH_C0 + f32(0.5)).astype(np.float32)
    s.sh_degree = sh_degree
    per = (sh_degree + 1) ** 2 - 1
    rest = np.empty((n, per, 3), np.float32)
    if sh_code_dim > 0 and per > 0:
        k = int(sh_code_dim)
        z = normal(stream_seed(seed, 7), k * n).reshape(n, k)
        basis = normal(stream_seed(seed, 8), k * per * 3).reshape(k, per * 3)
        basis *= f32(0.08) / np.sqrt(np.sum(basis * basis, axis=0, keepdims=True) + f32(1e-12))
        rest[:] = (z @ basis).astype(np.float32).reshape(n, per, 3)
    else:
        for c in range(per):
            rest[:, c, :] = (f32(0.08) * normal(stream_seed(seed, 7 + c), 3 * n)).reshape(n, 3)
    s.sh_rest = rest
    return s.finalize()


def lattice_view(scene: Scene, yaw_deg: float = 30.0, pitch_deg: float = 20.0):
    """The single orbit view of the small lattice workload."""
    c, r = scene.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.yaw = to_radians(yaw_deg)
    cam.pitch = to_radians(pitch_deg)
    return cam.view()


def orbit_camera(scene: Scene, distance: float = 12.0) -> OrbitCamera:
    """Orbit of the 1.2M-splat workload: target 0, given distance, FOV 50
    degrees, up -y; near plane from the scene's robust radius."""
    c, r = scene.bounds()
    cam = OrbitCamera.new(c, r, UpAxis.NEG_Y)
    cam.target = np.zeros(3, np.float32)
    cam.distance = f32(distance)
    cam.home = (cam.target.copy(), cam.distance, cam.yaw, cam.pitch)
    return cam


def orbit_views(cam: OrbitCamera, frames: int, warmup: int):
    """The bench orbit of ``src/bench.rs:51-71``: the home view, `warmup`
    views stepping yaw by 0.05, then `frames` views stepping yaw by
    2*pi/frames with pitch = 0.4 sin(0.1 i)."""
    home = cam.view()
    warm = []
    for _ in range(warmup):
        cam.rotate(0.05, 0.0)
        warm.append(cam.view())
    timed = []
    for i in range(frames):
        cam.rotate(f32(2.0 * np.pi) / f32(frames), 0.0)
        cam.pitch = f32(0.4) * f32(np.sin(f32(i) * f32(0.1)))
        timed.append(cam.view())
    return home, warm, timed


BATCH_SIZES = [(160, 96), (320, 192), (640, 360), (1280, 720), (1920, 1080), (3840, 2160)]


def batch_scenes(sizes=(50_000, 400_000, 3_000_000), degrees=(0, 1, 3), seed: int = 0x5EED0B00):
    """The batching workload's scenes: cluster scenes with the 1.2M workload's
    distributions, separate seeds (seed + index)."""
    return [cluster_scene(n, seed=seed + i, sh_degree=d) for i, (n, d) in enumerate(zip(sizes, degrees))]


def batch_views(scenes, n_views: int = 96, seed: int = 0x5EED0B96, sizes=BATCH_SIZES):
    """n_views (scene index, view, width, height) over `scenes`: scene uniform,
    resolution uniform from `sizes`, yaw U[0, 2 pi), pitch U[-0.6, 0.6], FOV
    U[40, 70] degrees, target 0 at distance 12, up -y."""
    u = uniform(seed, 5 * n_views).reshape(n_views, 5)
    out = []
    cams = [orbit_camera(s) for s in scenes]
    for i in range(n_views):
        k = min(int(u[i, 0] * len(scenes)), len(scenes) - 1)
        w, h = sizes[min(int(u[i, 1] * len(sizes)), len(sizes) - 1)]
        base = cams[k]
        cam = OrbitCamera(base.target.copy(), base.distance, f32(u[i, 2] * f32(2.0 * np.pi)),
                          f32(u[i, 3] * f32(1.2) - f32(0.6)), to_radians(f32(40.0) + f32(30.0) * u[i, 4]), base.up,
                          base.scene_radius)
        out.append((k, cam.view(), w, h))
    return out
