"""The allocation-free PCG entry point (drape_cuda_pcg_noalloc), for callers that cannot allocate device memory: a
host whose device memory belongs to another framework's pool, or a frame-paced loop that may not call
cudaMalloc/cudaFree. It runs the same kernels as drape_cuda_pcg with all scratch in one file-scope device array.

Called through the C ABI on device buffers the test owns (torch allocates them; the entry point itself allocates
nothing), twice in a row, and compared with the allocating entry point drape_cuda_pcg within the tests' PCG
tolerance. This file is collected last, so a run that stops at its first failure has already run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from drape_b200 import scenes as S

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_kernels.npz")
pytestmark = pytest.mark.gpu


def _float4(a):
    a = np.asarray(a, np.float32).reshape(-1, 3)
    out = np.zeros((len(a), 4), np.float32)
    out[:, :3] = a
    return out


def _systems(oracle_mod):
    G = np.load(GOLDEN)
    n = len(G["rig_row_start"]) - 1
    rig = dict(row_start=G["rig_row_start"], col_index=G["rig_col_index"], blocks=G["rig_blocks"].reshape(-1, 9),
               pinned=G["rig_pinned"], active=np.zeros(n, np.uint8), normals=np.zeros((n, 3), np.float32),
               grad=(-G["rig_b"]).astype(np.float32), max_it=50, tol=1e-2)
    scene = S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50)
    scene.garments[0].initial_positions[:, 1] -= 0.147
    o = oracle_mod.OracleSolver()
    o.build(scene)
    for _ in range(3):
        o.step(1 / 60, 1, 2)
    sysm = o.capture_system(1 / 60)
    sheet = dict(row_start=sysm["row_start"], col_index=sysm["col_index"],
                 blocks=sysm["blocks"].reshape(-1, 9).astype(np.float32),
                 pinned=np.zeros(len(sysm["diag_slot"]), np.uint8), active=sysm["active"],
                 normals=sysm["normals"].astype(np.float32), grad=sysm["grad"].astype(np.float32), max_it=50,
                 tol=1e-2)
    return {"rig": rig, "sheet": sheet}


def _noalloc(gpu, sysd):
    import torch
    dev = torch.device("cuda", 0)
    n = len(sysd["row_start"]) - 1
    slots = int(sysd["row_start"][-1])
    sp = (slots + 31) // 32 * 32
    planes = np.zeros((9, sp), np.float32)
    planes[:, :slots] = sysd["blocks"].T
    t = {
        "row_start": torch.tensor(sysd["row_start"].astype(np.int64), dtype=torch.int32, device=dev),
        "col_index": torch.tensor(sysd["col_index"].astype(np.int64), dtype=torch.int32, device=dev),
        "blocks": torch.tensor(planes, device=dev),
        "pinned": torch.tensor(sysd["pinned"], dtype=torch.uint8, device=dev),
        "active": torch.tensor(sysd["active"], dtype=torch.uint8, device=dev),
        "normals": torch.tensor(_float4(sysd["normals"]), device=dev),
        "grad": torch.tensor(_float4(sysd["grad"]), device=dev),
        "step": torch.full((n, 4), float("nan"), device=dev),
        "resid": torch.full((n, 4), float("nan"), device=dev),
        "iterations": torch.full((1,), -7, dtype=torch.int32, device=dev),
    }
    L = gpu.load()
    stream = torch.cuda.current_stream(dev)
    code = L.drape_cuda_pcg_noalloc(n, slots, t["row_start"].data_ptr(), t["col_index"].data_ptr(),
                                    t["blocks"].data_ptr(), sp, t["pinned"].data_ptr(), t["active"].data_ptr(),
                                    t["normals"].data_ptr(), t["grad"].data_ptr(), sysd["max_it"], sysd["tol"],
                                    t["step"].data_ptr(), t["resid"].data_ptr(), t["iterations"].data_ptr(),
                                    C.c_void_p(stream.cuda_stream))
    assert code == 0, L.drape_cuda_last_error(None)
    torch.cuda.synchronize(dev)
    return (t["step"][:, :3].cpu().numpy(), t["resid"][:, :3].cpu().numpy(), int(t["iterations"].item()))


@pytest.mark.parametrize("name", ["rig", "sheet"])
def test_noalloc_pcg_matches_allocating_entry_point_twice(gpu, oracle_mod, name):
    sysd = _systems(oracle_mod)[name]
    ref_step, ref_resid, ref_its = gpu.pcg(sysd["row_start"], sysd["col_index"], sysd["blocks"], sysd["pinned"],
                                           sysd["active"], sysd["normals"], sysd["grad"], sysd["max_it"], sysd["tol"])
    for _ in range(2):  # the second call sees the scratch the first one left behind
        step, resid, its = _noalloc(gpu, sysd)
        assert its == ref_its
        assert np.linalg.norm(step - ref_step) <= 1e-6 * np.linalg.norm(ref_step)
        assert np.linalg.norm(resid - ref_resid) <= 1e-6 * np.linalg.norm(ref_resid)


def test_noalloc_rejects_systems_beyond_its_scratch(gpu):
    L = gpu.load()
    too_many = 8192 + 1
    code = L.drape_cuda_pcg_noalloc(too_many, 0, 1, 1, 1, 32, 1, None, None, 1, 10, 1e-2, 1, 1, 1, None)
    assert code == gpu.INVALID
    assert b"8192" in L.drape_cuda_last_error(None)
    code = L.drape_cuda_pcg_noalloc(16, 131072 + 1, 1, 1, 1, 131072 + 32, 1, None, None, 1, 10, 1e-2, 1, 1, 1, None)
    assert code == gpu.INVALID
    assert b"131072" in L.drape_cuda_last_error(None)
