"""Builds the sm_100a rasterizer library ``splat_b200/libsplat_cuda.so`` in-tree.

Each CUDA source compiles with nvcc for ``sm_100a`` only; the projection
translation unit additionally gets ``--fmad=false`` so its f32 arithmetic is
the reference's unfused x86 arithmetic, bit for bit. Objects go to
``splat_b200/_build``; the shared library links the CUDA runtime statically
and exports only the C ABI of ``include/splat_cuda.h``.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsplat_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
                 "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
SOURCES = {
    "api.cu": [],
    "project.cu": ["--fmad=false"],
    "binning.cu": [],
    "blend.cu": [],
    "noalloc.cu": [],
    "batch.cu": [],
    "mlp.cu": [],
    "decode.cu": ["--fmad=false"],
    "term.cu": [],
    "shard.cu": [],
}
HEADERS = [os.path.join(CSRC, "common.cuh"), os.path.join(CSRC, "tilesort.cuh"), os.path.join(CSRC, "handle.h"),
           os.path.join(CSRC, "umma.cuh"), os.path.join(CSRC, "mlp.cuh"), os.path.join(CSRC, "sh.cuh"),
           os.path.join(CSRC, "geom.cuh"),
           os.path.join(ROOT, "include", "splat_cuda.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(obj)
        if _stale(obj, [path] + HEADERS) or ptxas_info:
            cmd = [NVCC] + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xcompiler", "-fvisibility=hidden"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
