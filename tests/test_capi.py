"""The C-ABI library loads, exports every symbol include/*.h declares, and fails loudly (no CPU fallback) where no
usable device exists. No compute calls here."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b((?:drape_cuda|drape_model|drape_precond|drape_batch|drape_bake|drape_mesh)_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("drape_cuda_create", "drape_cuda_build", "drape_cuda_step", "drape_cuda_read_positions",
                     "drape_cuda_stats", "drape_cuda_snapshot", "drape_cuda_restore", "drape_cuda_set_phase",
                     "drape_cuda_update_fabric", "drape_cuda_range", "drape_cuda_particle_count"):
        assert required in names


def test_library_exports_every_declared_symbol(cuda_mod):
    path = cuda_mod.library_path()
    lib = C.CDLL(path)
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T ((?:drape_cuda|drape_model|drape_precond|drape_batch|drape_bake|drape_mesh)_\w+)", out))
    assert set(declared_functions()) <= exported


def test_library_is_built_for_sm100a(cuda_mod):
    out = subprocess.run(["cuobjdump", "--list-elf", cuda_mod.library_path()], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_no_device_is_a_loud_error(cuda_mod):
    """Without a usable device, creating a solver fails with DRAPE_DEVICE_ERROR and a "cuda: ..." message."""
    if cuda_mod.is_available():
        pytest.skip("a device is present")
    with pytest.raises(cuda_mod.CudaError, match="cuda"):
        cuda_mod.CudaSolver(0)


def test_null_handle_errors(cuda_mod):
    from drape_b200 import batch
    B = batch._lib()
    assert B.drape_batch_step(None, 1 / 60, 1, 2) == cuda_mod.INVALID
    assert B.drape_batch_build(None) == cuda_mod.INVALID
    L = cuda_mod.load()
    assert L.drape_cuda_step(None, 1 / 60, 1, 2) == cuda_mod.INVALID
    assert L.drape_cuda_build(None, None) == cuda_mod.INVALID
    assert L.drape_cuda_version() >= 100
