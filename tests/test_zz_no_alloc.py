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


def _noalloc(gpu, sysd, slots=None):
    """Runs drape_cuda_pcg_noalloc on device copies of `sysd`; `slots` overrides the slot count passed by value (the
    structure checks compare it with row_start[n]). Returns (step, resid, iterations written on the device)."""
    import torch
    dev = torch.device("cuda", 0)
    n = len(sysd["row_start"]) - 1
    if slots is None:
        slots = int(sysd["row_start"][-1])
    slots = int(slots)
    stored = len(sysd["blocks"])
    sp = (max(slots, stored) + 31) // 32 * 32
    planes = np.zeros((9, sp), np.float32)
    planes[:, :stored] = sysd["blocks"].T
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


def _tiled(sysd, tiles):
    """`tiles` block-diagonal copies of a system (each copy's columns shifted by its row offset), each copy's gradient
    scaled differently so the copies do not solve identical problems."""
    rs, ci = sysd["row_start"].astype(np.int64), sysd["col_index"].astype(np.int64)
    n1, b1 = len(rs) - 1, len(ci)
    scale = np.repeat(1.0 + 0.25 * np.arange(tiles), n1)[:, None]
    return dict(row_start=np.concatenate([rs[:-1] + t * b1 for t in range(tiles)] + [np.array([tiles * b1])]).astype(
                    np.uint32),
                col_index=np.concatenate([ci + t * n1 for t in range(tiles)]).astype(np.uint32),
                blocks=np.tile(sysd["blocks"], (tiles, 1)), pinned=np.tile(sysd["pinned"], tiles),
                active=np.tile(sysd["active"], tiles), normals=np.tile(sysd["normals"], (tiles, 1)),
                grad=(np.tile(sysd["grad"], (tiles, 1)) * scale).astype(np.float32), max_it=sysd["max_it"],
                tol=sysd["tol"])


def test_noalloc_near_its_size_limit_matches_allocating_entry_point(gpu, oracle_mod):
    """Five copies of the sheet system: 8,000 of the 8,192 rows and ~99k of the 131,072 block slots, so the work
    vectors, the column region and the partials behind it are all used close to their ends."""
    sysd = _tiled(_systems(oracle_mod)["sheet"], 5)
    n, slots = len(sysd["row_start"]) - 1, int(sysd["row_start"][-1])
    assert 7000 < n <= 8192 and slots <= 131072
    ref_step, ref_resid, ref_its = gpu.pcg(sysd["row_start"], sysd["col_index"], sysd["blocks"], sysd["pinned"],
                                           sysd["active"], sysd["normals"], sysd["grad"], sysd["max_it"], sysd["tol"])
    for _ in range(2):
        step, resid, its = _noalloc(gpu, sysd)
        assert its == ref_its
        assert np.linalg.norm(step - ref_step) <= 1e-6 * np.linalg.norm(ref_step)
        assert np.linalg.norm(resid - ref_resid) <= 1e-6 * np.linalg.norm(ref_resid)


def _broken(sysd, kind):
    d = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in sysd.items()}
    rs, ci = d["row_start"].astype(np.int64), d["col_index"].astype(np.uint32)
    n = len(rs) - 1
    i = n // 2
    if kind == "row_without_diagonal":
        row = np.arange(rs[i], rs[i + 1])
        k = row[ci[row] == i][0]
        ci[k] = ci[row[0]] if ci[row[0]] != i else ci[row[-1]]  # the diagonal's column replaced by a neighbour's
    elif kind == "column_out_of_range":
        ci[rs[i]] = n + 10
    elif kind == "row_start_decreasing":
        rs[i], rs[i + 1] = rs[i + 1], rs[i]
    elif kind == "row_start_past_slots":
        rs[-1] += 40
    d["row_start"], d["col_index"] = rs.astype(np.uint32), ci
    slots = int(sysd["row_start"][-1])
    return d, slots


@pytest.mark.parametrize("kind", ["row_without_diagonal", "column_out_of_range", "row_start_decreasing",
                                  "row_start_past_slots"])
def test_noalloc_refuses_inconsistent_structure_then_recovers(gpu, oracle_mod, kind):
    """A structure the allocating entry point would reject is refused on the device: the iteration output is -2 and
    step/resid keep their contents (NaN here), with every access of the check kept in bounds. The next valid call
    gives the allocating entry point's result again."""
    sysd = _systems(oracle_mod)["rig"]
    bad, slots = _broken(sysd, kind)
    step, resid, its = _noalloc(gpu, bad, slots=slots)
    assert its == -2
    assert np.isnan(step).all() and np.isnan(resid).all()
    ref_step, _, ref_its = gpu.pcg(sysd["row_start"], sysd["col_index"], sysd["blocks"], sysd["pinned"],
                                   sysd["active"], sysd["normals"], sysd["grad"], sysd["max_it"], sysd["tol"])
    step, _, its = _noalloc(gpu, sysd)
    assert its == ref_its
    assert np.linalg.norm(step - ref_step) <= 1e-6 * np.linalg.norm(ref_step)


def test_noalloc_refuses_fewer_slots_than_rows(gpu):
    L = gpu.load()
    code = L.drape_cuda_pcg_noalloc(16, 15, 1, 1, 1, 32, 1, None, None, 1, 10, 1e-2, 1, 1, 1, None)
    assert code == gpu.INVALID
