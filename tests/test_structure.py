"""Bit-exact integer artefacts, checked on the CPU: the product's host model builder (libdrape_cuda.so,
drape_model_build: sort-based) against the oracle's literal restatement of SimModel::build / buildStructure
(std::map edge order, per-row sorted vectors, lower_bound slots; sim_model.cpp:35-175)."""
import ctypes as C

import numpy as np
import pytest

from drape_b200 import scenes as S
from drape_b200.scene import Scene, SceneDesc, drape_scene_desc, jersey_fabric

KEYS = ["row_start", "col_index", "diag_slot", "stretch_slots", "hinge_slots", "seam_slots", "stretch_v", "hinge_v",
        "seam_ab"]


def product_structure(cuda_mod, scene):
    L = cuda_mod.load()
    L.drape_model_build.argtypes = [C.POINTER(drape_scene_desc), C.POINTER(C.c_void_p)]
    L.drape_model_destroy.argtypes = [C.c_void_p]
    L.drape_model_last_error.restype = C.c_char_p
    L.drape_model_structure_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.drape_model_structure.argtypes = [C.c_void_p] + [C.POINTER(C.c_uint32)] * 9
    desc = SceneDesc(scene)
    h = C.c_void_p()
    code = L.drape_model_build(desc.ptr(), C.byref(h))
    if code != 0:
        cuda_mod._raise(code, L.drape_model_last_error())
    try:
        sz = (C.c_uint32 * 5)()
        assert L.drape_model_structure_sizes(h, sz) == 0
        n, B, Sn, H, K = list(sz)
        out = dict(row_start=np.zeros(n + 1, np.uint32), col_index=np.zeros(B, np.uint32),
                   diag_slot=np.zeros(n, np.uint32), stretch_slots=np.zeros((Sn, 9), np.uint32),
                   hinge_slots=np.zeros((H, 16), np.uint32), seam_slots=np.zeros((K, 4), np.uint32),
                   stretch_v=np.zeros((Sn, 3), np.uint32), hinge_v=np.zeros((H, 4), np.uint32),
                   seam_ab=np.zeros((K, 2), np.uint32))
        assert L.drape_model_structure(h, *[out[k].ctypes.data_as(C.POINTER(C.c_uint32)) for k in KEYS]) == 0
        return out
    finally:
        L.drape_model_destroy(h)


SCENES = {
    "sheet_40x40": lambda: S.sheet_on_sphere(),
    "sewn_pair": lambda: Scene([S.sewn_pair()]),
    "strip": lambda: S.strip_scene(),
    "tube_10k": lambda: S.tube_10k(field=S.sphere_field()),
    "tube_variant": lambda: S.tube_variant(3, 6000, field_n=16),
    "two_garments": lambda: Scene([S.flat_garment("a", 0.1, 0.1, 0.02, jersey_fabric()), S.sewn_pair()]),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_structure_bit_exact(cuda_mod, oracle_mod, name):
    scene = SCENES[name]()
    p = product_structure(cuda_mod, scene)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    ref = o.structure()
    for k in KEYS:
        assert p[k].shape == ref[k].shape, k
        assert np.array_equal(p[k], ref[k]), k


def test_structure_invariants(cuda_mod):
    scene = S.tube_10k(field=S.sphere_field())
    p = product_structure(cuda_mod, scene)
    rs, ci, ds = p["row_start"], p["col_index"], p["diag_slot"]
    n = len(ds)
    for i in range(n):
        row = ci[rs[i]:rs[i + 1]]
        assert np.all(np.diff(row.astype(np.int64)) > 0)  # sorted unique
        assert ci[ds[i]] == i
    # every slot of a term addresses (v[a], v[b])
    for vs, slots, N in ((p["stretch_v"], p["stretch_slots"], 3), (p["hinge_v"], p["hinge_slots"], 4),
                         (p["seam_ab"], p["seam_slots"], 2)):
        for a in range(N):
            for b in range(N):
                s = slots[:, a * N + b]
                assert np.all(ci[s] == vs[:, b])
                assert np.all((s >= rs[vs[:, a]]) & (s < rs[vs[:, a] + 1]))
    # the hinge count: interior edges of both panels plus one seam hinge per consecutive seam pair
    nx, ny = 63, 80
    edges = (nx - 1) * ny + nx * (ny - 1) + (nx - 1) * (ny - 1)
    interior = edges - 2 * (nx - 1) - 2 * (ny - 1)
    assert len(p["hinge_v"]) == 2 * interior + 2 * (ny - 1)


def test_hinge_order_is_map_order(oracle_mod):
    """Interior hinges appear in lexicographic (min, max) edge order, as std::map iterates (sim_model.cpp:124-146)."""
    scene = Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())])
    o = oracle_mod.OracleSolver()
    o.build(scene)
    hv = o.structure()["hinge_v"]
    keys = [(min(e0, e1), max(e0, e1)) for e0, e1 in hv[:, 2:4]]
    assert keys == sorted(keys)


def test_gather_lists_follow_reference_order(oracle_mod):
    """gpu_solver_core.cpp:184-224: per particle the own term, then stretch, hinge and seam contributions in term order."""
    scene = Scene([S.sewn_pair()])
    o = oracle_mod.OracleSolver()
    o.build(scene)
    st = o.structure()
    n, Sn, H = len(st["diag_slot"]), len(st["stretch_v"]), len(st["hinge_v"])
    gs, gi = st["grad_start"], st["grad_idx"]
    for i in range(n):
        lst = gi[gs[i]:gs[i + 1]]
        assert lst[0] == i
        assert np.all(np.diff(lst.astype(np.int64)) > 0)
        expected = 1 + (st["stretch_v"] == i).sum() + (st["hinge_v"] == i).sum() + (st["seam_ab"] == i).sum()
        assert len(lst) == expected


@pytest.mark.parametrize("bad,exc", [("pin", IndexError), ("force", IndexError), ("triangle", ValueError)])
def test_build_errors_match_reference(cuda_mod, oracle_mod, bad, exc):
    """build throws std::out_of_range for pins/forces out of range (sim_model.cpp:184, :190) and std::invalid_argument
    for an inconsistent mesh."""
    g = S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())
    scene = Scene([g])
    if bad == "pin":
        scene.pins.append((10_000, (0.0, 0.0, 0.0)))
    elif bad == "force":
        scene.forces.append((10_000, (0.0, 0.0, 0.0)))
    else:
        g.triangles = g.triangles.copy()
        g.triangles[0, 0] = 10_000
    with pytest.raises(exc):
        product_structure(cuda_mod, scene)
    if bad != "triangle":
        with pytest.raises(exc):
            oracle_mod.OracleSolver().build(scene)


def product_gather_lists(cuda_mod, scene):
    """The product's gather lists (drape_model_gather_lists) re-expressed in the reference's contribution numbering:
    per particle [i, then the term-gradient index of each incidence entry]; per block slot [i for a diagonal slot,
    then the term-block index of each contribution] (gpu_solver_core.cpp:184-224)."""
    L = cuda_mod.load()
    L.drape_model_build.argtypes = [C.POINTER(drape_scene_desc), C.POINTER(C.c_void_p)]
    L.drape_model_destroy.argtypes = [C.c_void_p]
    L.drape_model_last_error.restype = C.c_char_p
    L.drape_model_gather_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.drape_model_gather_lists.argtypes = [C.c_void_p] + [C.POINTER(C.c_uint32)] * 5
    desc = SceneDesc(scene)
    h = C.c_void_p()
    code = L.drape_model_build(desc.ptr(), C.byref(h))
    if code != 0:
        cuda_mod._raise(code, L.drape_model_last_error())
    try:
        sz = (C.c_uint32 * 4)()
        assert L.drape_model_gather_sizes(h, sz) == 0
        n, E, O, NC = list(sz)
        inc_start, inc_entry = np.zeros(n + 1, np.uint32), np.zeros(E, np.uint32)
        off_slot, off_start, off_contrib = np.zeros(O, np.uint32), np.zeros(O + 1, np.uint32), np.zeros(NC, np.uint32)
        arrs = [inc_start, inc_entry, off_slot, off_start, off_contrib]
        assert L.drape_model_gather_lists(h, *[a.ctypes.data_as(C.POINTER(C.c_uint32)) for a in arrs]) == 0
    finally:
        L.drape_model_destroy(h)
    return inc_start, inc_entry, off_slot, off_start, off_contrib


@pytest.mark.parametrize("name", ["sheet_40x40", "sewn_pair", "tube_variant", "two_garments"])
def test_assembly_gather_lists_match_reference(cuda_mod, oracle_mod, name):
    """Bit-exact: every gradient row and every block slot of the product's assembly sums the same contributions in the
    same order as the reference's gather lists (the oracle's restatement of gpu_solver_core.cpp:184-224)."""
    scene = SCENES[name]()
    inc_start, inc_entry, off_slot, off_start, off_contrib = product_gather_lists(cuda_mod, scene)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    st = o.structure()
    n, Sn, H = len(st["diag_slot"]), len(st["stretch_v"]), len(st["hinge_v"])
    kind, term, a = inc_entry >> 30, (inc_entry >> 2) & 0x0FFFFFFF, (inc_entry & 3).astype(np.int64)
    term = term.astype(np.int64)
    # Reference numbering: gradients n + 3t + a | n + 3S + 4h + a | n + 3S + 4H + 2k + a; blocks n + 9t + 3a + b |
    # n + 9S + 16h + 4a + b | n + 9S + 16H + 4k + 2a + b.
    gbase = np.where(kind == 0, n + 3 * term, np.where(kind == 1, n + 3 * Sn + 4 * term, n + 3 * Sn + 4 * H + 2 * term))
    grad_ref = gbase + a
    arity = np.where(kind == 0, 3, np.where(kind == 1, 4, 2))
    bbase = np.where(kind == 0, n + 9 * term, np.where(kind == 1, n + 9 * Sn + 16 * term, n + 9 * Sn + 16 * H + 4 * term))
    for i in range(n):
        e0, e1 = inc_start[i], inc_start[i + 1]
        got = [i] + list(grad_ref[e0:e1])
        ref = list(st["grad_idx"][st["grad_start"][i]:st["grad_start"][i + 1]])
        assert got == ref, i
    B = len(st["col_index"])
    per_slot = [None] * B
    for i in range(n):  # diagonal slots: the own term, then block (a, a) of every incidence entry
        e = np.arange(inc_start[i], inc_start[i + 1])
        per_slot[st["diag_slot"][i]] = [i] + list(bbase[e] + arity[e] * a[e] + a[e])
    rs = st["row_start"]
    for k in range(len(off_slot)):
        row, t = int(off_slot[k]) >> 6, int(off_slot[k]) & 63
        c = off_contrib[off_start[k]:off_start[k + 1]].astype(np.int64)
        e, b = c >> 2, c & 3
        per_slot[rs[row] + t] = list(bbase[e] + arity[e] * a[e] + b)
    for s in range(B):
        ref = list(st["block_idx"][st["block_start"][s]:st["block_start"][s + 1]])
        assert per_slot[s] == ref, s
