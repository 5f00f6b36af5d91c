"""Orbit camera and resolved view, mirroring the reference's ``src/camera.rs``.

Camera space follows the 3DGS/COLMAP convention (x right, y down, z
forward), as in ``camera.rs:1-2``. All arithmetic is binary32 (numpy
float32 scalars) in the reference's operation order.
"""

from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field

import numpy as np

f32 = np.float32
PI = f32(math.pi)
TAU = f32(2.0 * math.pi)


def to_radians(deg) -> np.float32:
    """``f32::to_radians``: deg * (PI / 180)."""
    return f32(deg) * (PI / f32(180.0))


def _v(x, y, z) -> np.ndarray:
    return np.array([x, y, z], dtype=np.float32)


def dot(a, b) -> np.float32:
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def cross(a, b) -> np.ndarray:
    # glam Vec3::cross
    return _v(a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0], a[0] * b[1] - b[0] * a[1])


def normalize(a) -> np.ndarray:
    inv = f32(1.0) / np.sqrt(dot(a, a))
    return (a * inv).astype(np.float32)


class UpAxis(enum.Enum):
    """World axis pointing up on screen (``camera.rs:8-66``)."""

    POS_Y = "+y"
    NEG_Y = "-y"
    POS_Z = "+z"
    NEG_Z = "-z"

    def vector(self) -> np.ndarray:
        return {UpAxis.POS_Y: _v(0, 1, 0), UpAxis.NEG_Y: _v(0, -1, 0), UpAxis.POS_Z: _v(0, 0, 1),
                UpAxis.NEG_Z: _v(0, 0, -1)}[self]

    def next(self) -> "UpAxis":
        return {UpAxis.NEG_Y: UpAxis.POS_Y, UpAxis.POS_Y: UpAxis.POS_Z, UpAxis.POS_Z: UpAxis.NEG_Z,
                UpAxis.NEG_Z: UpAxis.NEG_Y}[self]

    def label(self) -> str:
        return self.value.upper()

    def horizontal(self):
        up = self.vector()
        seed = _v(0, 0, 1) if abs(up[1]) > 0.5 else _v(0, 1, 0)
        a = normalize(cross(seed, up))
        b = normalize(cross(up, a))
        return a, b

    @staticmethod
    def parse(s: str) -> "UpAxis":
        t = s.lower()
        table = {"+y": UpAxis.POS_Y, "y": UpAxis.POS_Y, "-y": UpAxis.NEG_Y, "+z": UpAxis.POS_Z, "z": UpAxis.POS_Z,
                 "-z": UpAxis.NEG_Z}
        if t not in table:
            raise ValueError(f"invalid up axis '{s}' (use +y, -y, +z or -z)")
        return table[t]


MAX_PITCH = f32(89.0) * PI / f32(180.0)


@dataclass
class View:
    """Resolved camera pose used by renderers (``camera.rs:161-187``)."""

    eye: np.ndarray
    right: np.ndarray
    down: np.ndarray
    forward: np.ndarray
    fov_y: np.float32
    near: np.float32

    def rotation(self) -> np.ndarray:
        """World-to-camera rotation; rows are right/down/forward."""
        return np.stack([self.right, self.down, self.forward]).astype(np.float32)

    def focal(self, height: int) -> np.float32:
        return (f32(height) * f32(0.5)) / f32(np.tan(f32(self.fov_y) * f32(0.5)))

    def to_camera(self, p) -> np.ndarray:
        d = np.asarray(p, np.float32) - self.eye
        return _v(dot(d, self.right), dot(d, self.down), dot(d, self.forward))

    def to_array(self) -> np.ndarray:
        """14 floats: eye, right, down, forward, fov_y, near (the C ABI's view)."""
        return np.concatenate([self.eye, self.right, self.down, self.forward,
                               np.array([self.fov_y, self.near], np.float32)]).astype(np.float32)

    @staticmethod
    def from_array(a) -> "View":
        a = np.asarray(a, np.float32)
        return View(a[0:3].copy(), a[3:6].copy(), a[6:9].copy(), a[9:12].copy(), f32(a[12]), f32(a[13]))

    @staticmethod
    def looking_along_z(eye, fov_deg=50.0, near=0.01) -> "View":
        """The fixed +z view the reference's image tests use (tests/render.rs:12-22)."""
        return View(np.asarray(eye, np.float32), _v(1, 0, 0), _v(0, 1, 0), _v(0, 0, 1), to_radians(fov_deg), f32(near))


@dataclass
class OrbitCamera:
    """Orbit camera (``camera.rs:68-159``)."""

    target: np.ndarray
    distance: np.float32
    yaw: np.float32
    pitch: np.float32
    fov_y: np.float32
    up: UpAxis
    scene_radius: np.float32
    home: tuple = field(default=None, repr=False)

    @staticmethod
    def new(center, radius, up: UpAxis = UpAxis.NEG_Y) -> "OrbitCamera":
        fov_y = to_radians(50.0)
        distance = f32(radius) / f32(np.tan(fov_y * f32(0.5))) * f32(1.1)
        pitch = to_radians(15.0)
        c = OrbitCamera(np.asarray(center, np.float32).copy(), distance, f32(0.0), pitch, fov_y, up, f32(radius))
        c.home = (c.target.copy(), distance, f32(0.0), pitch)
        c.reset()
        return c

    def reset(self):
        t, d, y, p = self.home
        self.target = t.copy()
        self.distance = d
        self.yaw = y
        self.pitch = p

    def rotate(self, dyaw, dpitch):
        y = f32(self.yaw + f32(dyaw))
        r = f32(np.fmod(y, TAU))
        self.yaw = f32(r + TAU) if r < 0 else r  # rem_euclid
        self.pitch = f32(min(max(f32(self.pitch + f32(dpitch)), -MAX_PITCH), MAX_PITCH))

    def zoom(self, factor):
        lo = self.scene_radius * f32(1e-3)
        hi = self.scene_radius * f32(1e3)
        self.distance = f32(min(max(f32(self.distance * f32(factor)), lo), hi))

    def pan(self, dx, dy):
        v = self.view()
        scale = self.distance * f32(np.tan(self.fov_y * f32(0.5))) * f32(2.0)
        self.target = (self.target + (v.right * f32(dx) + v.down * f32(dy)) * scale).astype(np.float32)

    def eye(self) -> np.ndarray:
        a, b = self.up.horizontal()
        up = self.up.vector()
        sy, cy = f32(np.sin(self.yaw)), f32(np.cos(self.yaw))
        sp, cp = f32(np.sin(self.pitch)), f32(np.cos(self.pitch))
        d = (a * sy + b * cy) * cp + up * sp
        return (self.target + d.astype(np.float32) * self.distance).astype(np.float32)

    def near(self) -> np.float32:
        return f32(max(self.scene_radius * f32(0.05), f32(1e-4)))

    def view(self) -> View:
        eye = self.eye()
        forward = normalize(self.target - eye)
        right = normalize(cross(forward, self.up.vector()))
        down = cross(forward, right)
        return View(eye, right, down, forward, self.fov_y, self.near())
