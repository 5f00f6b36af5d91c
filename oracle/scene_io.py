"""ORACLE — test infrastructure only.

Restatement of the reference's scene file readers and writers, for checking
the device-side decoders (``splat_cuda_create_from_splat`` /
``splat_cuda_create_from_ply``): ``src/splat_format.rs:18-64`` (the 32-byte
``.splat`` record) and ``src/ply.rs:104-430`` (3DGS PLY, ascii and binary
little / big endian). ``parse_*`` return an un-finalized
``splat_b200.scene.Scene`` with the reference's f32 arithmetic; f32 ``exp``
and ``ln`` are evaluated in double and rounded once (the correctly rounded
f32 result). Only tests import this module.
"""

from __future__ import annotations

import numpy as np

from splat_b200.scene import Scene

f32 = np.float32
SH_C0 = f32(0.2820948)  # src/sh.rs:5

_TYPES = {"char": "b", "int8": "b", "uchar": "B", "uint8": "B", "short": "h", "int16": "h", "ushort": "H",
          "uint16": "H", "int": "i", "int32": "i", "uint": "I", "uint32": "I", "float": "f", "float32": "f",
          "double": "d", "float64": "d"}


def exp32(x):
    return np.exp(np.asarray(x, np.float64)).astype(np.float32)


def ln32(x):
    return np.log(np.asarray(x, np.float64)).astype(np.float32)


def sigmoid32(x):
    """src/scene.rs:180-184 in f32."""
    return (f32(1.0) / (f32(1.0) + exp32(-np.asarray(x, np.float32)))).astype(np.float32)


def logit32(p):
    """src/scene.rs:186-191 in f32."""
    p = np.clip(np.asarray(p, np.float32), f32(1e-6), f32(1.0 - 1e-6))
    return ln32(p / (f32(1.0) - p))


# --- .splat (src/splat_format.rs) ------------------------------------------------

def write_splat(s: Scene) -> bytes:
    """splat_format::write (src/splat_format.rs:46-64)."""
    n = len(s)
    q = np.asarray(s.rotations, np.float32)
    sq = q * q
    ln = np.sqrt((sq[:, 0] + sq[:, 2]) + (sq[:, 1] + sq[:, 3]))
    qn = q / ln[:, None]

    def u8c(v):
        return np.clip(np.round(np.asarray(v, np.float32) * f32(255.0)), 0, 255).astype(np.uint8)

    def qc(v):
        return np.clip(np.round(np.asarray(v, np.float32) * f32(128.0) + f32(128.0)), 0, 255).astype(np.uint8)

    rec = np.zeros((n, 32), np.uint8)
    rec[:, 0:24] = np.concatenate([np.asarray(s.positions, "<f4"), np.asarray(s.scales, "<f4")], 1).view(np.uint8)
    rec[:, 24:27] = u8c(s.colors)
    rec[:, 27] = u8c(s.opacities)
    rec[:, 28] = qc(qn[:, 3])
    rec[:, 29:32] = qc(qn[:, 0:3])
    return rec.tobytes()


def parse_splat(data: bytes) -> Scene:
    """splat_format::parse (src/splat_format.rs:18-44)."""
    if len(data) % 32:
        raise ValueError(f".splat file size {len(data)} is not a multiple of 32 bytes")
    r = np.frombuffer(data, np.uint8).reshape(-1, 32)
    s = Scene()
    fl = r[:, 0:24].copy().view("<f4").astype(np.float32)
    s.positions = fl[:, 0:3].copy()
    s.scales = np.abs(fl[:, 3:6])
    s.colors = (r[:, 24:27].astype(np.float32) / f32(255.0)).astype(np.float32)
    s.opacities = (r[:, 27].astype(np.float32) / f32(255.0)).astype(np.float32)
    qv = (r[:, 28:32].astype(np.float32) - f32(128.0)) / f32(128.0)
    s.rotations = np.stack([qv[:, 1], qv[:, 2], qv[:, 3], qv[:, 0]], 1).astype(np.float32)
    s.sh_degree = 0
    return s


# --- PLY (src/ply.rs) -------------------------------------------------------------

def write_ply(s: Scene, fmt: str = "binary_little_endian", types=None) -> bytes:
    """ply::write (src/ply.rs:381-430) in the 3DGS layout; `fmt` may also be
    binary_big_endian or ascii, `types` maps property names to PLY scalar types
    (default float) to exercise the reader's conversions."""
    types = types or {}
    n = len(s)
    per = s.rest_per_splat()
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"]
    names += [f"f_rest_{i}" for i in range(per * 3)]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    cols = {}
    p = np.asarray(s.positions, np.float32)
    dc = ((np.asarray(s.colors, np.float32) - f32(0.5)) / SH_C0).astype(np.float32)
    rest = np.asarray(s.sh_rest, np.float32).reshape(n, per, 3)
    for k, nm in enumerate("xyz"):
        cols[nm] = p[:, k]
    for nm in ("nx", "ny", "nz"):
        cols[nm] = np.zeros(n, np.float32)
    for k in range(3):
        cols[f"f_dc_{k}"] = dc[:, k]
    for c in range(3):
        for i in range(per):
            cols[f"f_rest_{c * per + i}"] = rest[:, i, c]
    cols["opacity"] = logit32(s.opacities)
    sc = np.maximum(np.asarray(s.scales, np.float32), f32(1e-12))
    for k in range(3):
        cols[f"scale_{k}"] = ln32(sc[:, k])
    q = np.asarray(s.rotations, np.float32)
    for k, j in enumerate((3, 0, 1, 2)):
        cols[f"rot_{k}"] = q[:, j]
    hdr = f"ply\nformat {fmt} 1.0\ncomment generated by splat-tui\nelement vertex {n}\n"
    for nm in names:
        hdr += f"property {types.get(nm, 'float')} {nm}\n"
    hdr += "end_header\n"
    if fmt == "ascii":
        rows = []
        for i in range(n):
            rows.append(" ".join(repr(float(cols[nm][i])) if _TYPES[types.get(nm, "float")] in "fd"
                                 else str(int(cols[nm][i])) for nm in names))
        return hdr.encode() + ("\n".join(rows) + "\n").encode()
    end = "<" if fmt == "binary_little_endian" else ">"
    rec = np.empty(n, np.dtype([(nm, end + _TYPES[types.get(nm, "float")]) for nm in names]))
    for nm in names:
        rec[nm] = cols[nm]
    return hdr.encode() + rec.tobytes()


def parse_ply(data: bytes) -> Scene:
    """ply::parse (src/ply.rs:218-379) for vertex-only files."""
    pos = data.find(b"end_header", 0, 1 << 20)
    if pos < 0:
        raise ValueError("PLY header missing end_header")
    body = data.index(b"\n", pos) + 1
    lines = data[:pos].decode().splitlines()
    if not lines or lines[0].strip() != "ply":
        raise ValueError("not a PLY file (missing 'ply' magic)")
    fmt, props, count = None, [], 0
    for ln in lines[1:]:
        w = ln.split()
        if not w or w[0] in ("comment", "obj_info"):
            continue
        if w[0] == "format":
            fmt = w[1]
        elif w[0] == "element":
            count = int(w[2])
        elif w[0] == "property":
            props.append((w[2], w[1]))
    names = [nm for nm, _ in props]
    idx = {nm: i for i, nm in enumerate(names)}
    if fmt == "ascii":
        vals = data[body:].split()
        rows = np.array([float(v) for v in vals[: count * len(props)]], np.float64).reshape(count, len(props))
    else:
        end = "<" if fmt == "binary_little_endian" else ">"
        dt = np.dtype([(nm, end + _TYPES[t]) for nm, t in props])
        if len(data) < body + dt.itemsize * count:
            raise ValueError("PLY body truncated")
        rec = np.frombuffer(data, dt, count, body)
        rows = np.stack([rec[nm].astype(np.float64) for nm, _ in props], 1) if count else np.zeros((0, len(props)))

    def col(nm):
        return rows[:, idx[nm]].astype(np.float32)

    s = Scene()
    s.positions = np.stack([col("x"), col("y"), col("z")], 1)
    if all(k in idx for k in ("f_dc_0", "f_dc_1", "f_dc_2")):
        s.colors = np.stack([col(f"f_dc_{k}") * SH_C0 + f32(0.5) for k in range(3)], 1).astype(np.float32)
    elif all(k in idx for k in ("red", "green", "blue")):
        scale = f32(1.0 / 255.0) if dict(props)["red"] in ("uchar", "uint8") else f32(1.0)
        s.colors = np.stack([col(c) * scale for c in ("red", "green", "blue")], 1).astype(np.float32)
    else:
        s.colors = np.full((count, 3), 0.8, np.float32)
    s.opacities = sigmoid32(col("opacity")) if "opacity" in idx else np.ones(count, np.float32)
    if all(f"scale_{k}" in idx for k in range(3)):
        s.scales = np.stack([exp32(col(f"scale_{k}")) for k in range(3)], 1)
    else:
        s.scales = np.full((count, 3), 0.01, np.float32)
    if all(f"rot_{k}" in idx for k in range(4)):
        s.rotations = np.stack([col("rot_1"), col("rot_2"), col("rot_3"), col("rot_0")], 1)
    else:
        s.rotations = np.tile(np.array([0, 0, 0, 1], np.float32), (count, 1))
    nrest = 0
    while f"f_rest_{nrest}" in idx:
        nrest += 1
    deg = {0: 0, 9: 1, 24: 2, 45: 3}.get(nrest, 0)
    per = (deg + 1) ** 2 - 1
    s.sh_degree = deg
    s.sh_rest = np.stack([np.stack([col(f"f_rest_{c * per + k}") for c in range(3)], 1) for k in range(per)], 1) \
        if per else np.zeros((count, 0, 3), np.float32)
    return s
