"""Build the in-tree CUDA library hitomi_b200/libhitomi_b200.so for sm_100a.

The library is a plain shared object with the C ABI declared in include/hitomi_gpu.h;
nothing in it links against torch.  nvcc cross-compiles it without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhitomi_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "hg_engine.cu"), os.path.join(HERE, "csrc", "hg_static.cu")]
HEADERS = [
    os.path.join(HERE, "csrc", f)
    for f in os.listdir(os.path.join(HERE, "csrc"))
    if f.endswith((".cuh", ".hpp", ".h"))
] + [os.path.join(ROOT, "include", "hitomi_gpu.h")]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [
        nvcc(),
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-O3", "-lineinfo", "-std=c++17",
        "-Xcompiler", "-fPIC", "-shared",
        "-I", os.path.join(ROOT, "include"),
        "-o", LIB + ".tmp",
    ] + SOURCES
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
