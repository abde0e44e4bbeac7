"""Builds libdrape_cuda.so in-tree for sm_100a with nvcc (no JIT cache: the library travels with the tree)."""
from __future__ import annotations

import os
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)          # drape-2_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
LIB_DIR = os.path.join(ROOT, "lib")
LIB = os.path.join(LIB_DIR, "libdrape_cuda.so")

SOURCES = ["solver.cu", "batch.cu", "learned.cu", "model.cpp"]
HEADERS = ["kernels.cuh", "device_math.cuh", "model.hpp", "learned.hpp", "umma.cuh", "device_model.hpp",
           "device_buffer.hpp", "solver_kernels.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files += [os.path.join(REPO, "include", h) for h in ("drape_cuda.h", "drape_scene.h", "drape_precond.h", "drape_batch.h")]
    return files


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the CUDA library if any source is newer than it; returns its path."""
    if not force and not stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-o", LIB + ".tmp"] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
