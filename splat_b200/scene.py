"""Gaussian scene in structure-of-arrays form, mirroring ``src/scene.rs``.

Parameters are *activated* (linear scales, unit quaternions, opacities in
[0, 1], base colour ``SH_C0 * f_dc + 0.5``), exactly what the reference's
``Scene`` holds (``scene.rs:11-28``). ``finalize`` sanitises and derives the
3D covariance upper triangle with glam's operation order
(``scene.rs:153-186, 261-270``).
"""

from __future__ import annotations

import numpy as np

f32 = np.float32

SH_C0 = f32(0.2820948)  # src/sh.rs:5


def coeffs_for_degree(degree: int) -> int:
    return (degree + 1) * (degree + 1)


def degree_from_rest_count(rest: int):
    for d in range(4):
        if 3 * (coeffs_for_degree(d) - 1) == rest:
            return d
    return None


def covariance(scales: np.ndarray, quats_xyzw: np.ndarray) -> np.ndarray:
    """R S Sᵀ Rᵀ upper triangle (xx, xy, xz, yy, yz, zz), vectorised, glam
    Mat3::from_quat and Mat3 * Mat3 order (``scene.rs:170-178``)."""
    s = np.asarray(scales, np.float32)
    q = np.asarray(quats_xyzw, np.float32)
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    x2, y2, z2 = x + x, y + y, z + z
    xx, xy, xz = x * x2, x * y2, x * z2
    yy, yz, zz = y * y2, y * z2, z * z2
    wx, wy, wz = w * x2, w * y2, w * z2
    one = f32(1.0)
    zero = np.zeros_like(x)
    # columns of R
    r0 = (one - (yy + zz), xy + wz, xz - wy)
    r1 = (xy - wz, one - (xx + zz), yz + wx)
    r2 = (xz + wy, yz - wx, one - (xx + yy))

    def mulv(c0, c1, c2, v):  # Mat3 * Vec3: c0*v.x, + c1*v.y, + c2*v.z
        return tuple((c0[k] * v[0] + c1[k] * v[1]) + c2[k] * v[2] for k in range(3))

    sx, sy, sz = s[:, 0], s[:, 1], s[:, 2]
    m0 = mulv(r0, r1, r2, (sx, zero, zero))
    m1 = mulv(r0, r1, r2, (zero, sy, zero))
    m2 = mulv(r0, r1, r2, (zero, zero, sz))
    # s = m * mᵀ; column j of mᵀ is row j of m.
    c = [mulv(m0, m1, m2, (m0[j], m1[j], m2[j])) for j in range(3)]
    return np.stack([c[0][0], c[1][0], c[2][0], c[1][1], c[2][1], c[2][2]], axis=1).astype(np.float32)


class Scene:
    """A collection of 3D gaussians with activated parameters."""

    def __init__(self):
        self.positions = np.zeros((0, 3), np.float32)
        self.scales = np.zeros((0, 3), np.float32)
        self.rotations = np.zeros((0, 4), np.float32)  # x, y, z, w
        self.opacities = np.zeros((0,), np.float32)
        self.colors = np.zeros((0, 3), np.float32)
        self.sh_degree = 0
        self.sh_rest = np.zeros((0, 0, 3), np.float32)
        self.cov3d = np.zeros((0, 6), np.float32)
        self._pending = None

    def __len__(self):
        return len(self.positions)

    def rest_per_splat(self) -> int:
        return coeffs_for_degree(self.sh_degree) - 1

    def push(self, pos, scale, rot_xyzw, opacity, color):
        """Append one gaussian (degree-0 colour), as ``Scene::push``."""
        if self._pending is None:
            self._pending = []
        self._pending.append((pos, scale, rot_xyzw, opacity, color))

    def _flush(self):
        if not self._pending:
            return
        p = self._pending
        self._pending = None
        self.positions = np.concatenate([self.positions, np.array([a[0] for a in p], np.float32).reshape(-1, 3)])
        self.scales = np.concatenate([self.scales, np.array([a[1] for a in p], np.float32).reshape(-1, 3)])
        self.rotations = np.concatenate([self.rotations, np.array([a[2] for a in p], np.float32).reshape(-1, 4)])
        self.opacities = np.concatenate([self.opacities, np.array([a[3] for a in p], np.float32)])
        self.colors = np.concatenate([self.colors, np.array([a[4] for a in p], np.float32).reshape(-1, 3)])

    def finalize(self) -> "Scene":
        """Validate, sanitise and derive cov3d (``scene.rs:153-186``)."""
        self._flush()
        n = len(self.positions)
        per = self.rest_per_splat()
        if self.sh_degree == 0:
            self.sh_rest = np.zeros((n, 0, 3), np.float32)
        if (len(self.scales) != n or len(self.rotations) != n or len(self.opacities) != n or len(self.colors) != n
                or self.sh_rest.reshape(-1, 3).shape[0] != n * per):
            raise ValueError("inconsistent scene arrays")
        self.sh_rest = np.ascontiguousarray(self.sh_rest.reshape(n, per, 3), np.float32)
        q = np.asarray(self.rotations, np.float32)
        # glam's SSE2 Quat::length: sqrt((x²+z²) + (y²+w²)); then q / len.
        sq = q * q
        length = np.sqrt((sq[:, 0] + sq[:, 2]) + (sq[:, 1] + sq[:, 3]))
        ok = np.isfinite(length) & (length > f32(1e-12))
        safe = np.where(ok, length, f32(1.0)).astype(np.float32)
        qn = (q / safe[:, None]).astype(np.float32)
        qn[~ok] = np.array([0, 0, 0, 1], np.float32)
        self.rotations = qn
        o = np.asarray(self.opacities, np.float32)
        self.opacities = np.where(np.isfinite(o), np.clip(o, f32(0.0), f32(1.0)), f32(0.0)).astype(np.float32)
        self.positions = np.ascontiguousarray(self.positions, np.float32)
        self.colors = np.ascontiguousarray(self.colors, np.float32)
        self.scales = np.ascontiguousarray(self.scales, np.float32)
        self.cov3d = covariance(self.scales, self.rotations) if n else np.zeros((0, 6), np.float32)
        return self

    def shard(self, s0: int, s1: int) -> "Scene":
        """Splats [s0, s1) of this finalized scene as a scene of their own
        (one device's share of a frame split by splats)."""
        self._flush()
        out = Scene()
        for name in ("positions", "scales", "rotations", "opacities", "colors", "sh_rest", "cov3d"):
            setattr(out, name, np.ascontiguousarray(getattr(self, name)[s0:s1]))
        out.sh_degree = self.sh_degree
        return out

    def bounds(self):
        """Robust centre/radius (``scene.rs:212-258``): per-axis median and
        min(p90, 2 * p50) of the distances, on a subsample of <= ~200k points."""
        if len(self.positions) == 0:
            return np.zeros(3, np.float32), f32(1.0)
        step = max(len(self.positions) // 200_000, 1)
        pts = self.positions[::step]
        pts = pts[np.all(np.isfinite(pts), axis=1)]
        if len(pts) == 0:
            return np.zeros(3, np.float32), f32(1.0)
        mid = len(pts) // 2
        center = np.array([np.partition(pts[:, k], mid)[mid] for k in range(3)], np.float32)
        d0 = pts - center
        d = np.sqrt((d0[:, 0] * d0[:, 0] + d0[:, 1] * d0[:, 1]) + d0[:, 2] * d0[:, 2]).astype(np.float32)

        def pct(q):
            idx = min(int(f32(len(d)) * f32(q)), len(d) - 1)
            return np.partition(d, idx)[idx]

        radius = f32(min(pct(0.9), f32(2.0) * pct(0.5)))
        return center, (radius if radius > f32(1e-6) else f32(1.0))

    def to_fp16(self) -> "HalfScene":
        """This scene with scales, rotations, opacities, base colours and SH
        stored as IEEE binary16 (round to nearest even); positions stay f32."""
        self._flush()
        return HalfScene.from_scene(self)


def _half_bits(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float32).astype(np.float16)).view(np.uint16)


class HalfScene:
    """FP16 parameter storage of a finalized scene: f32 positions (12 B), f16
    scales (6 B), rotations x, y, z, w (8 B), opacity (2 B) and base colour +
    SH rest, RGB innermost ((rest + 1) * 3 halves): 124 bytes per degree-3
    splat against 232 for the f32 scene. The device forms the 3D covariance
    from the decoded scale and rotation."""

    def __init__(self, positions, scales, rotations, opacities, sh, sh_degree: int):
        self.positions = np.ascontiguousarray(positions, np.float32)
        self.scales = np.ascontiguousarray(scales, np.uint16)
        self.rotations = np.ascontiguousarray(rotations, np.uint16)
        self.opacities = np.ascontiguousarray(opacities, np.uint16)
        self.sh = np.ascontiguousarray(sh, np.uint16)  # n x (rest + 1) x 3
        self.sh_degree = int(sh_degree)

    @classmethod
    def from_scene(cls, s: Scene) -> "HalfScene":
        n = len(s)
        per = s.rest_per_splat()
        sh = np.concatenate([np.asarray(s.colors, np.float32).reshape(n, 1, 3),
                             np.asarray(s.sh_rest, np.float32).reshape(n, per, 3)], axis=1)
        return cls(s.positions, _half_bits(s.scales), _half_bits(s.rotations), _half_bits(s.opacities),
                   _half_bits(sh), s.sh_degree)

    def __len__(self):
        return len(self.positions)

    def shard(self, s0: int, s1: int) -> "HalfScene":
        """Splats [s0, s1) as a scene of their own (one device's share)."""
        return HalfScene(self.positions[s0:s1], self.scales[s0:s1], self.rotations[s0:s1], self.opacities[s0:s1],
                         self.sh[s0:s1], self.sh_degree)

    def decoded(self) -> dict:
        """The stored values widened back to f32 (exact), as arrays named like
        Scene's: positions, scales, rotations (x, y, z, w; as stored, not
        renormalised), opacities, colors, sh_rest, sh_degree."""
        n = len(self)
        h = lambda a: a.view(np.float16).astype(np.float32)  # noqa: E731
        sh = h(self.sh).reshape(n, -1, 3)
        return {"positions": self.positions, "scales": h(self.scales).reshape(n, 3),
                "rotations": h(self.rotations).reshape(n, 4), "opacities": h(self.opacities).reshape(n),
                "colors": np.ascontiguousarray(sh[:, 0, :]), "sh_rest": np.ascontiguousarray(sh[:, 1:, :]),
                "sh_degree": self.sh_degree}

    def decoded_scene(self) -> Scene:
        """The decoded values as a finalized f32 Scene: rotation normalisation,
        opacity clamp and covariance exactly as the device applies them to
        the stored halves."""
        d = self.decoded()
        s = Scene()
        s.positions = d["positions"].copy()
        s.scales = d["scales"]
        s.rotations = d["rotations"]
        s.opacities = d["opacities"]
        s.colors = d["colors"]
        s.sh_degree = self.sh_degree
        s.sh_rest = d["sh_rest"]
        return s.finalize()
