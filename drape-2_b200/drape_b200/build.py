"""Builds libdrape_cuda.so in-tree for sm_100a with nvcc (no JIT cache: the library travels with the tree)."""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)          # drape-2_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
LIB_DIR = os.path.join(ROOT, "lib")
LIB = os.path.join(LIB_DIR, "libdrape_cuda.so")
OBJ_DIR = os.path.join(LIB_DIR, "obj")

SOURCES = ["solver.cu", "batch.cu", "learned.cu", "bake.cu", "model.cpp", "mesher.cpp"]
HEADERS = ["kernels.cuh", "device_math.cuh", "model.hpp", "learned.hpp", "umma.cuh", "device_model.hpp",
           "device_buffer.hpp", "solver_kernels.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _inputs():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    headers = ("drape_cuda.h", "drape_scene.h", "drape_precond.h", "drape_batch.h", "drape_bake.h", "drape_mesh.h")
    files += [os.path.join(REPO, "include", h) for h in headers]
    return files


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the CUDA library if any source is newer than it (each source to an object in parallel, then one
    link); returns its path."""
    if not force and not stale():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        subprocess.run([NVCC, *flags, "-c", os.path.join(CSRC, src), "-o", obj], check=True, cwd=CSRC)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as pool:
        objs = list(pool.map(compile_one, SOURCES))
    subprocess.run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB + ".tmp", *objs], check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
