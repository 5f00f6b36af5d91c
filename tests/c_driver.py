"""Builds tests/abi_driver.c (a plain C99 host of the C ABI) against
include/splat_cuda.h and the in-tree library."""

import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(out_dir: str) -> str:
    exe = os.path.join(out_dir, "abi_driver")
    lib_dir = os.path.join(ROOT, "splat_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_driver.c"), "-o", exe, "-L", lib_dir, "-lsplat_cuda",
                    f"-Wl,-rpath,{lib_dir}", "-lm"], check=True, capture_output=True, text=True)
    return exe
