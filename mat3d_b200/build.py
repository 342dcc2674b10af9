"""Build recipe for the native libraries of mat3d_b200 (in-tree, sm_100a).

    python -m mat3d_b200.build          # libmat3d_b200.so (CUDA solver + C ABI + C++ drop-in classes)

The shared library is written next to this file so that it travels with the
source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmat3d_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]

SOURCES = [os.path.join(CSRC, "solver.cu"), os.path.join(CSRC, "noalloc.cu"), os.path.join(CSRC, "compat.cpp"),
           os.path.join(CSRC, "batch.cpp"), os.path.join(CSRC, "serve.cpp"),
           os.path.join(CSRC, "solver2d.cu"), os.path.join(CSRC, "rec.cu"), os.path.join(CSRC, "rec_compat.cpp")]
DEPS = SOURCES + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
    os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]


def _nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isabs(p) and os.path.exists(p) or not os.path.isabs(p)):
            return p
    return "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = True) -> str:
    if not force and not needs_build():
        return LIB
    srcs = [s for s in SOURCES if os.path.exists(s)]
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB, *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
