"""Test scenes: small seeded workloads plus restatements of the reference's
procedural test scenes (``src/gen.rs``: cube, galaxy, shballs) used by its
agreement tests (``tests/render.rs:45-76``). The restatements keep each
scene's structure and sizes; values are not bit-identical to the Rust
generator (glam/libm details), which the tests do not need: both renderers
always consume the same arrays.
"""

from __future__ import annotations

import numpy as np

from splat_b200.scene import Scene
from splat_b200 import synth

f32 = np.float32


def _quat_rot_x(angle):
    h = angle * 0.5
    return np.array([np.sin(h), 0, 0, np.cos(h)], np.float32)


def _quat_mul(a, b):
    ax, ay, az, aw = a[..., 0], a[..., 1], a[..., 2], a[..., 3]
    bx, by, bz, bw = b[..., 0], b[..., 1], b[..., 2], b[..., 3]
    return np.stack([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz], -1).astype(np.float32)


def _arc_quat(frm, to):
    """Quat::from_rotation_arc for unit vectors (vectorised)."""
    to = np.atleast_2d(to).astype(np.float64)
    frm = np.broadcast_to(np.asarray(frm, np.float64), to.shape)
    d = np.sum(frm * to, -1)
    c = np.cross(frm, to)
    w = 1.0 + d
    q = np.concatenate([c, w[:, None]], -1)
    anti = w < 1e-6
    if np.any(anti):
        q[anti] = np.array([1.0, 0, 0, 0])
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    return q.astype(np.float32)


def _rot_z(angle):
    angle = np.asarray(angle, np.float64)
    return np.stack([np.zeros_like(angle), np.zeros_like(angle), np.sin(angle / 2), np.cos(angle / 2)], -1).astype(
        np.float32)


def _disc(n, radius, thickness, spin):
    q = _quat_mul(_arc_quat([0, 0, 1], n), _rot_z(spin))
    n_ = len(q)
    sc = np.stack([np.broadcast_to(radius, n_), np.broadcast_to(radius, n_), np.broadcast_to(thickness, n_)], -1)
    return sc.astype(np.float32), q


def _to_y_down(s: Scene):
    r = _quat_rot_x(np.pi)
    p = s.positions
    s.positions = np.stack([p[:, 0], -p[:, 1], -p[:, 2]], -1).astype(np.float32)
    s.rotations = _quat_mul(np.broadcast_to(r, s.rotations.shape), s.rotations)


def cube() -> Scene:
    """gen.rs:106-129: a 12^3 RGB lattice plus a 41x41 checker floor of discs."""
    n = 12
    step = 2.0 / (n - 1)
    idx = np.arange(n, dtype=np.float32)
    i, j, k = np.meshgrid(idx, idx, idx, indexing="ij")
    t = np.stack([i.ravel(), j.ravel(), k.ravel()], -1) / f32(n - 1)
    pos = t * 2 - 1
    m = len(pos)
    s = Scene()
    gi, gj = np.meshgrid(np.arange(-20, 21), np.arange(-20, 21), indexing="ij")
    gi, gj = gi.ravel(), gj.ravel()
    fpos = np.stack([gi * 0.12, np.full(gi.shape, -1.4), gj * 0.12], -1).astype(np.float32)
    shade = np.where((gi + gj) % 2 == 0, 0.85, 0.35).astype(np.float32)
    fsc, fq = _disc(np.tile([0.0, 1.0, 0.0], (len(gi), 1)), 0.07, 0.005, np.zeros(len(gi)))
    s.positions = np.concatenate([pos, fpos]).astype(np.float32)
    s.scales = np.concatenate([np.full((m, 3), step * 0.28, np.float32), fsc])
    s.rotations = np.concatenate([np.tile([0, 0, 0, 1], (m, 1)).astype(np.float32), fq])
    s.opacities = np.concatenate([np.full(m, 0.95, np.float32), np.full(len(gi), 0.9, np.float32)])
    s.colors = np.concatenate([t, np.repeat(shade[:, None], 3, 1)]).astype(np.float32)
    _to_y_down(s)
    return s.finalize()


def galaxy(n_stars=90_000, n_bulge=8_000, n_dust=6_000, seed=42) -> Scene:
    """gen.rs:160-205: log-spiral arms, a glowing bulge and dark dust discs."""
    rng = np.random.default_rng(seed)
    arms = 4
    arm = rng.integers(0, arms, n_stars).astype(np.float32)
    r = rng.random(n_stars) ** 0.6 * 3.0 + 0.05
    theta = arm / arms * 2 * np.pi + np.log(r) * 2.2 + rng.normal(size=n_stars) * 0.25 / (0.3 + r)
    h = rng.normal(size=n_stars) * 0.06 * (1.0 + 0.5 / (r + 0.2))
    spos = np.stack([r * np.cos(theta), h, r * np.sin(theta)], -1)
    heat = np.exp(-r * 0.9)[:, None]
    col = (np.array([0.55, 0.65, 1.0]) * (1 - heat) + np.array([1.0, 0.85, 0.55]) * heat) * rng.uniform(0.6, 1.2, (
        n_stars, 1))
    ssc = np.repeat(rng.uniform(0.006, 0.018, (n_stars, 1)), 3, 1)
    sop = rng.uniform(0.5, 1.0, n_stars)
    u = rng.normal(size=(n_bulge, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    bpos = u * np.abs(rng.normal(size=(n_bulge, 1))) * 0.35 * np.array([1.0, 0.5, 1.0])
    bcol = np.stack([np.ones(n_bulge), rng.uniform(0.75, 0.9, n_bulge), rng.uniform(0.45, 0.6, n_bulge)], -1)
    bsc = np.repeat(rng.uniform(0.02, 0.06, (n_bulge, 1)), 3, 1)
    darm = rng.integers(0, arms, n_dust).astype(np.float32)
    dr = rng.uniform(0.4, 2.6, n_dust)
    dth = darm / arms * 2 * np.pi + np.log(dr) * 2.2 - 0.25
    dpos = np.stack([dr * np.cos(dth), rng.normal(size=n_dust) * 0.01, dr * np.sin(dth)], -1)
    dsc, dq = _disc(np.tile([0.0, 1.0, 0.0], (n_dust, 1)), rng.uniform(0.04, 0.09, n_dust), 0.008,
                    rng.uniform(0, 2 * np.pi, n_dust))
    s = Scene()
    s.positions = np.concatenate([spos, bpos, dpos]).astype(np.float32)
    s.scales = np.concatenate([ssc, bsc, dsc]).astype(np.float32)
    ident = np.tile([0, 0, 0, 1], (n_stars + n_bulge, 1)).astype(np.float32)
    s.rotations = np.concatenate([ident, dq])
    s.opacities = np.concatenate([sop, np.full(n_bulge, 0.35), np.full(n_dust, 0.25)]).astype(np.float32)
    s.colors = np.concatenate([col, bcol, np.tile([0.12, 0.07, 0.05], (n_dust, 1))]).astype(np.float32)
    _to_y_down(s)
    return s.finalize()


def shballs(per_ball=12_000, seed=11) -> Scene:
    """gen.rs:257-293: three spheres of discs with degree-1/2/3 SH colour."""
    rng = np.random.default_rng(seed)
    centers = [(-1.2, 0.0, 0.0), (0.0, 0.0, 0.0), (1.2, 0.0, 0.0)]
    pos, sc, q, rest = [], [], [], []
    for kind, c in enumerate(centers):
        n = rng.normal(size=(per_ball, 3))
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        d_sc, d_q = _disc(n, 0.035, 0.006, rng.uniform(0, 2 * np.pi, per_ball))
        pos.append(np.asarray(c) + n * 0.5)
        sc.append(d_sc)
        q.append(d_q)
        r = np.zeros((per_ball, 15, 3), np.float32)
        if kind == 0:
            r[:, 2] = (-0.9, 0.6, 0.6)
        elif kind == 1:
            r[:, 5] = (0.9, -0.3, -0.6)
            r[:, 7] = (-0.4, 0.8, -0.2)
        else:
            r[:, 0] = (0.2, -0.2, 0.0)
            r[:, 9] = (0.0, 1.2, -1.2)
            r[:, 13] = (1.2, -0.6, 0.0)
            r[:, 14] = (-0.6, 0.0, 1.0)
        rest.append(r)
    s = Scene()
    s.positions = np.concatenate(pos).astype(np.float32)
    s.scales = np.concatenate(sc)
    s.rotations = np.concatenate(q)
    m = len(s.positions)
    s.opacities = np.full(m, 0.95, np.float32)
    s.colors = np.full((m, 3), 0.5, np.float32)
    s.sh_degree = 3
    s.sh_rest = np.concatenate(rest)
    _to_y_down(s)
    return s.finalize()


def clusters(n=20_000, seed=7, sh_degree=3) -> Scene:
    return synth.cluster_scene(n, seed=seed, sh_degree=sh_degree)


def splats(items) -> Scene:
    """tests/render.rs:24-31: isotropic, identity-rotation splats from
    (position, scale, opacity, colour) tuples."""
    s = Scene()
    for p, scale, op, c in items:
        s.push(p, (scale, scale, scale), (0, 0, 0, 1), op, c)
    return s.finalize()


def empty() -> Scene:
    return Scene().finalize()


def needles(n=20_000, seed=5, length=4.0, thickness=1e-4) -> Scene:
    """Long, thin splats close to the camera at the origin looking along +z:
    their projected 2D covariances are nearly rank one with entries ~1e7, so
    the f32 determinant a*c - b^2 cancels and some fall below 1e-6 (the FP16
    storage path's FP64 conic case)."""
    rng = np.random.default_rng(seed)
    s = Scene()
    z = rng.uniform(0.5, 3.0, n)
    xy = rng.uniform(-0.6, 0.6, (n, 2)) * z[:, None]
    s.positions = np.stack([xy[:, 0], xy[:, 1], z], 1).astype(np.float32)
    s.scales = np.tile(np.array([length, thickness, thickness], np.float32), (n, 1))
    s.rotations = rng.normal(size=(n, 4)).astype(np.float32)
    s.opacities = rng.uniform(0.3, 1.0, n).astype(np.float32)
    s.colors = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    return s.finalize()


def planes(n_big=20_000, n_small=20_000, seed=13, depths=(5.0, 6.0)) -> Scene:
    """Splats on planes facing a camera at the origin that looks along +z
    (View.looking_along_z): every splat of a plane has the same depth bits
    (t.z = 0 x + 0 y + 1 z exactly), so each tile's pairs fall into a few
    runs of equal depth that only the splat index orders (the reference's
    fix_ties, src/render/cpu.rs:396-414). Large splats crowd the centre, so
    central tiles hold tens of thousands of pairs, outer tiles hundreds."""
    rng = np.random.default_rng(seed)
    n = n_big + n_small
    z = np.asarray(depths, np.float32)[rng.integers(0, len(depths), n)]
    xy = np.concatenate([rng.normal(0.0, 0.4, (n_big, 2)), rng.uniform(-3.0, 3.0, (n_small, 2))])
    s = Scene()
    s.positions = np.stack([xy[:, 0] * z / 5.0, xy[:, 1] * z / 5.0, z], 1).astype(np.float32)
    sig = np.concatenate([rng.uniform(0.25, 0.6, n_big), rng.uniform(0.01, 0.05, n_small)])
    s.scales = np.stack([sig, sig * rng.uniform(0.5, 1.0, n), np.full(n, 0.01)], 1).astype(np.float32)
    ang = rng.uniform(0, np.pi, n)
    s.rotations = np.stack([np.zeros(n), np.zeros(n), np.sin(ang / 2), np.cos(ang / 2)], 1).astype(np.float32)
    s.opacities = rng.uniform(0.05, 0.6, n).astype(np.float32)
    s.colors = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    return s.finalize()
