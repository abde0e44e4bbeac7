"""ORACLE — test infrastructure only.

ctypes access to the two CPU checkers:
  OracleSolver   the FP64 restatement of the reference's CpuSolver (oracle/_build/liboracle.so; modes: faithful float
                 state, or full FP64), following libs/sim/src/cpu_solver.cpp and sim_model.cpp;
  RefEmulated    the reference's own FP32 kernel bodies (libs/sim/kernels/kernels.h, term_math.h) and EmulatedDevice,
                 compiled from the reference sources into oracle/_ref/libref_emulated.so, driven in the order of the
                 reference's GpuSolverCore.
Only tests, the smoke check and the benchmark's CPU-baseline leg import this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "drape-2_b200"))

from drape_b200.scene import (SceneDesc, drape_counters, drape_fabric, drape_field_desc,  # noqa: E402
                              drape_scene_desc, drape_stats, field_desc)

LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref_emulated.so")

_P = C.POINTER
_d, _f, _u8, _u32, _i32 = C.c_double, C.c_float, C.c_uint8, C.c_uint32, C.c_int32


def build(ref: bool = False) -> None:
    """Compiles the oracle (and, with ref and the reference sources present, oracle/_ref) with make."""
    targets = ["all"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _np(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a, ctype):
    return a.ctypes.data_as(_P(ctype))


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_int]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_last_error.argtypes = [C.c_void_p]
        L.oracle_build.argtypes = [C.c_void_p, _P(drape_scene_desc)]
        L.oracle_step.argtypes = [C.c_void_p, _d, C.c_int, C.c_int]
        L.oracle_set_phase.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.oracle_update_fabric.argtypes = [C.c_void_p, C.c_char_p, _P(drape_fabric), _u32]
        L.oracle_range.argtypes = [C.c_void_p, C.c_char_p, _P(_u32), _P(_u32)]
        L.oracle_particle_count.restype = C.c_size_t
        L.oracle_particle_count.argtypes = [C.c_void_p]
        L.oracle_read_positions.argtypes = [C.c_void_p, _P(_d), C.c_size_t]
        L.oracle_read_velocities.argtypes = [C.c_void_p, _P(_d), C.c_size_t]
        L.oracle_stats.argtypes = [C.c_void_p, _P(drape_stats)]
        L.oracle_counters.argtypes = [C.c_void_p, _P(drape_counters)]
        L.oracle_reset_counters.argtypes = [C.c_void_p]
        L.oracle_snapshot_sizes.argtypes = [C.c_void_p, _P(_u32), _P(_u32), _P(_u32)]
        L.oracle_snapshot.argtypes = [C.c_void_p, _P(_f), _P(_f), _P(_i32), _P(_d), _P(_f), _P(_d)]
        L.oracle_restore.argtypes = [C.c_void_p, _P(_f), _P(_f), _u32, _P(_i32), _P(_d), _u32, _P(_f), _u32, _P(_d), _u32]
        L.oracle_structure_sizes.argtypes = [C.c_void_p, _P(_u32)]
        L.oracle_structure.argtypes = [C.c_void_p] + [_P(_u32)] * 13
        L.oracle_term_constants.argtypes = [C.c_void_p, _P(_d), _P(_d), _P(_d), _P(_d)]
        L.oracle_contact_candidates.argtypes = [C.c_void_p, _P(_d), _P(_u8), _P(_d), _P(_d)]
        L.oracle_capture_system.argtypes = [C.c_void_p, _d, _P(_d), _P(_d), _P(_u8), _P(_d), _P(_d)]
        L.oracle_eval_stretch.argtypes = [_P(_d), _P(_d), _d, _P(drape_fabric), _d, _P(_d), _P(_d), _P(_d)]
        L.oracle_eval_hinge.argtypes = [_P(_d), _d, _d, _P(_d), _P(_d), _P(_d)]
        L.oracle_eval_seam.argtypes = [_P(_d), _d, _d, _P(_d), _P(_d), _P(_d)]
        L.oracle_eval_friction.argtypes = [_P(_d), _P(_d), _P(_d), _d, _d, _P(_d), _P(_d), _P(_d)]
        L.oracle_dihedral.restype = _d
        L.oracle_dihedral.argtypes = [_P(_d), _P(_d)]
        L.oracle_bending_coefficients.argtypes = [_d, _d, _P(_d), _P(_d)]
        L.oracle_edge_bend_stiffness.restype = _d
        L.oracle_edge_bend_stiffness.argtypes = [_d, _d, _P(_d), _P(_d)]
        L.oracle_field_sample.restype = _d
        L.oracle_field_sample.argtypes = [_P(drape_field_desc), _P(_d)]
        L.oracle_field_gradient.argtypes = [_P(drape_field_desc), _P(_d), _P(_d)]
        L.oracle_collide_body.argtypes = [_P(drape_field_desc), _f, _f, _P(_f), _P(_f)]
        L.oracle_land_on_body.argtypes = [_P(drape_field_desc), _f, _P(_f), _P(_f), _P(_f)]
        L.oracle_pcg.argtypes = [_u32, _P(_u32), _P(_u32), _P(_d), _P(_u8), _P(_u8), _P(_d), _P(_d), C.c_int, _d,
                                 _P(_d), _P(_d), _P(C.c_int)]
        from drape_b200.bake import drape_bake_options, drape_mesh_desc
        L.oracle_bake.argtypes = [_P(drape_mesh_desc), _u32, _P(drape_bake_options), _P(_d), _P(_i32)]
        L.oracle_bake_values.argtypes = [_P(_f), C.c_size_t]
        L.oracle_bake_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def bake(components, cell_size: float = 0.004, padding: float = 0.05, band: float = 0.02):
    """bakeCollisionField restated serially on the CPU (bake_impl.hpp): returns a scene.Field. Raises ValueError for
    an open component, as the reference throws std::invalid_argument."""
    from drape_b200.bake import MeshArray, drape_bake_options
    from drape_b200.scene import Field
    L = lib()
    arr = MeshArray(components)
    opts = drape_bake_options(cell_size, padding, band)
    origin, dims = (_d * 3)(), (_i32 * 3)()
    code = L.oracle_bake(arr.descs, arr.count, C.byref(opts), origin, dims)
    if code != 0:
        raise (ValueError if code == -1 else RuntimeError)(L.oracle_bake_last_error().decode())
    d = tuple(int(x) for x in dims)
    values = np.zeros(d[0] * d[1] * d[2], np.float32)
    if L.oracle_bake_values(_p(values, _f), values.size) != 0:
        raise RuntimeError("oracle bake values")
    return Field(np.array(origin[:]), float(cell_size), d, float(band), values.reshape(d[2], d[1], d[0]))


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError("oracle/_ref/libref_emulated.so is not built (needs the reference sources)")
        L = C.CDLL(REF_LIB)
        L.ref_create.restype = C.c_void_p
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_last_error.restype = C.c_char_p
        L.ref_last_error.argtypes = [C.c_void_p]
        L.ref_build.argtypes = [C.c_void_p, _P(drape_scene_desc)]
        L.ref_step.argtypes = [C.c_void_p, _d, C.c_int, C.c_int]
        L.ref_set_phase.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.ref_read_positions.argtypes = [C.c_void_p, _P(_d), C.c_size_t]
        L.ref_stats.argtypes = [C.c_void_p, _P(drape_stats)]
        L.ref_counters.argtypes = [C.c_void_p, _P(drape_counters)]
        L.ref_contact_setup.argtypes = [C.c_void_p, _P(_f), _P(_u8), _P(_f), _P(_f)]
        L.ref_eval_stretch.argtypes = [_P(_f), _P(_f), _f, _P(drape_fabric), _f, _P(_f), _P(_f), _P(_f)]
        L.ref_eval_hinge.argtypes = [_P(_f), _f, _f, _P(_f), _P(_f), _P(_f)]
        L.ref_eval_seam.argtypes = [_P(_f), _f, _f, _P(_f), _P(_f), _P(_f)]
        L.ref_eval_friction.argtypes = [_P(_f), _P(_f), _f, _f, _P(_f), _P(_f), _P(_f)]
        L.ref_field_sample.restype = _f
        L.ref_field_sample.argtypes = [_P(drape_field_desc), _P(_f)]
        L.ref_field_gradient.argtypes = [_P(drape_field_desc), _P(_f), _P(_f)]
        L.ref_collide_body.argtypes = [_P(drape_field_desc), _f, _f, _P(_f), _P(_f)]
        L.ref_land_on_body.argtypes = [_P(drape_field_desc), _f, _P(_f), _P(_f), _P(_f)]
        L.ref_invert_spd3.restype = C.c_int
        L.ref_invert_spd3.argtypes = [_P(_f), _P(_f)]
        L.ref_reduce.restype = _f
        L.ref_reduce.argtypes = [_P(_f), _u32]
        L.ref_pcg.argtypes = [_u32, _P(_u32), _P(_u32), _P(_f), _P(_u8), _P(_u8), _P(_f), _P(_f), C.c_int, _f,
                              _P(_f), _P(_f), _P(C.c_int)]
        _ref = L
    return _ref


class OracleError(RuntimeError):
    pass


def _raise(code, msg):
    if code == 0:
        return
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    if code == -1:
        raise ValueError(msg)
    if code == -2:
        raise IndexError(msg)
    raise OracleError(msg)


class OracleSolver:
    """The Solver interface (libs/sim/include/drape/sim/solver.hpp:85-98) over the CPU restatement."""

    def __init__(self, full_fp64: bool = False):
        self.L = lib()
        self.h = self.L.oracle_create(1 if full_fp64 else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    def _check(self, code):
        _raise(code, self.L.oracle_last_error(self.h))

    def build(self, scene):
        self._desc = SceneDesc(scene)
        self._check(self.L.oracle_build(self.h, self._desc.ptr()))

    def step(self, dt=1.0 / 60.0, substeps=2, iterations=2):
        self._check(self.L.oracle_step(self.h, dt, substeps, iterations))

    def set_phase(self, garment, phase):
        self._check(self.L.oracle_set_phase(self.h, garment.encode(), int(phase)))

    def update_fabric(self, garment, fabrics):
        arr = (drape_fabric * len(fabrics))(*[f.to_c() for f in fabrics])
        self._check(self.L.oracle_update_fabric(self.h, garment.encode(), arr, len(fabrics)))

    def range(self, garment):
        off, cnt = _u32(), _u32()
        self._check(self.L.oracle_range(self.h, garment.encode(), C.byref(off), C.byref(cnt)))
        return off.value, cnt.value

    def particle_count(self):
        return int(self.L.oracle_particle_count(self.h))

    def positions(self):
        n = self.particle_count()
        out = np.zeros((n, 3))
        self._check(self.L.oracle_read_positions(self.h, _p(out, _d), n))
        return out

    def velocities(self):
        n = self.particle_count()
        out = np.zeros((n, 3))
        self._check(self.L.oracle_read_velocities(self.h, _p(out, _d), n))
        return out

    def stats(self):
        st = drape_stats()
        self._check(self.L.oracle_stats(self.h, C.byref(st)))
        return st

    def counters(self):
        c = drape_counters()
        self.L.oracle_counters(self.h, C.byref(c))
        return c

    def reset_counters(self):
        self.L.oracle_reset_counters(self.h)

    def snapshot(self):
        n, g, k = _u32(), _u32(), _u32()
        self._check(self.L.oracle_snapshot_sizes(self.h, C.byref(n), C.byref(g), C.byref(k)))
        n, g, k = n.value, g.value, k.value
        snap = dict(positions=np.zeros((n, 3), np.float32), velocities=np.zeros((n, 3), np.float32),
                    phases=np.zeros(g, np.int32), assembly_time=np.zeros(g), seam_start_gap=np.zeros(k, np.float32),
                    contact_force=np.zeros(n))
        self._check(self.L.oracle_snapshot(self.h, _p(snap["positions"], _f), _p(snap["velocities"], _f),
                                           _p(snap["phases"], _i32), _p(snap["assembly_time"], _d),
                                           _p(snap["seam_start_gap"], _f), _p(snap["contact_force"], _d)))
        return snap

    def restore(self, snap):
        pos = _np(snap["positions"], np.float32)
        vel = _np(snap["velocities"], np.float32)
        ph = _np(snap["phases"], np.int32)
        at = _np(snap["assembly_time"], np.float64)
        sg = _np(snap["seam_start_gap"], np.float32)
        cf = _np(snap["contact_force"], np.float64)
        self._check(self.L.oracle_restore(self.h, _p(pos, _f), _p(vel, _f), len(pos), _p(ph, _i32), _p(at, _d),
                                          len(ph), _p(sg, _f), len(sg), _p(cf, _d), len(cf)))

    def structure(self):
        sz = (_u32 * 7)()
        self._check(self.L.oracle_structure_sizes(self.h, sz))
        n, B, S, H, K, G, BB = list(sz)
        out = dict(row_start=np.zeros(n + 1, np.uint32), col_index=np.zeros(B, np.uint32),
                   diag_slot=np.zeros(n, np.uint32), stretch_slots=np.zeros((S, 9), np.uint32),
                   hinge_slots=np.zeros((H, 16), np.uint32), seam_slots=np.zeros((K, 4), np.uint32),
                   stretch_v=np.zeros((S, 3), np.uint32), hinge_v=np.zeros((H, 4), np.uint32),
                   seam_ab=np.zeros((K, 2), np.uint32), grad_start=np.zeros(n + 1, np.uint32),
                   grad_idx=np.zeros(G, np.uint32), block_start=np.zeros(B + 1, np.uint32),
                   block_idx=np.zeros(BB, np.uint32))
        keys = ["row_start", "col_index", "diag_slot", "stretch_slots", "hinge_slots", "seam_slots", "stretch_v",
                "hinge_v", "seam_ab", "grad_start", "grad_idx", "block_start", "block_idx"]
        self._check(self.L.oracle_structure(self.h, *[_p(out[k], _u32) for k in keys]))
        return out

    def term_constants(self):
        st = self.structure()
        S, H, n = len(st["stretch_v"]), len(st["hinge_v"]), len(st["diag_slot"])
        dm, area, hk, mass = np.zeros((S, 4)), np.zeros(S), np.zeros(H), np.zeros(n)
        self._check(self.L.oracle_term_constants(self.h, _p(dm, _d), _p(area, _d), _p(hk, _d), _p(mass, _d)))
        return dict(stretch_dm_inv=dm, stretch_area=area, hinge_k=hk, mass=mass)

    def contact_candidates(self, x):
        x = _np(x, np.float64)
        n = len(x)
        near, nrm, off = np.zeros(n, np.uint8), np.zeros((n, 3)), np.zeros(n)
        self._check(self.L.oracle_contact_candidates(self.h, _p(x, _d), _p(near, _u8), _p(nrm, _d), _p(off, _d)))
        return near, nrm, off

    def capture_system(self, h):
        st = self.structure()
        n, B = len(st["diag_slot"]), len(st["col_index"])
        blocks, grad, active, normals, e = np.zeros((B, 3, 3)), np.zeros((n, 3)), np.zeros(n, np.uint8), \
            np.zeros((n, 3)), _d()
        self._check(self.L.oracle_capture_system(self.h, h, _p(blocks, _d), _p(grad, _d), _p(active, _u8),
                                                 _p(normals, _d), C.byref(e)))
        return dict(blocks=blocks, grad=grad, active=active, normals=normals, energy=e.value, **st)


def pcg(row_start, col_index, blocks, pinned, active, normals, grad, max_iterations=50, tolerance=1e-2):
    """CpuSolver::solveLinear on a given system (cpu_solver.cpp:169-213)."""
    L = lib()
    n = len(row_start) - 1
    rs, ci = _np(row_start, np.uint32), _np(col_index, np.uint32)
    bl = _np(blocks, np.float64).reshape(-1, 9)
    pn, ac = _np(pinned, np.uint8), _np(active, np.uint8)
    nm, g = _np(normals, np.float64), _np(grad, np.float64)
    step, resid, its = np.zeros((n, 3)), np.zeros((n, 3)), C.c_int()
    code = L.oracle_pcg(n, _p(rs, _u32), _p(ci, _u32), _p(bl, _d), _p(pn, _u8), _p(ac, _u8), _p(nm, _d), _p(g, _d),
                        max_iterations, tolerance, _p(step, _d), _p(resid, _d), C.byref(its))
    _raise(code, "oracle_pcg failed")
    return step, resid, its.value


class RefEmulated:
    """The reference's FP32 GPU algorithm run on its own EmulatedDevice (oracle/_ref)."""

    def __init__(self):
        self.L = ref()
        self.h = self.L.ref_create()

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    def _check(self, code):
        _raise(code, self.L.ref_last_error(self.h))

    def build(self, scene):
        self._desc = SceneDesc(scene)
        self._n = scene.particle_count
        self._check(self.L.ref_build(self.h, self._desc.ptr()))

    def step(self, dt=1.0 / 60.0, substeps=2, iterations=2):
        self._check(self.L.ref_step(self.h, dt, substeps, iterations))

    def set_phase(self, garment, phase):
        self._check(self.L.ref_set_phase(self.h, garment.encode(), int(phase)))

    def positions(self):
        out = np.zeros((self._n, 3))
        self._check(self.L.ref_read_positions(self.h, _p(out, _d), self._n))
        return out

    def stats(self):
        st = drape_stats()
        self._check(self.L.ref_stats(self.h, C.byref(st)))
        return st

    def counters(self):
        c = drape_counters()
        self.L.ref_counters(self.h, C.byref(c))
        return c

    def contact_setup(self, x_start):
        xs = _np(x_start, np.float32)
        n = len(xs)
        near, nrm, off = np.zeros(n, np.uint8), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self._check(self.L.ref_contact_setup(self.h, _p(xs, _f), _p(near, _u8), _p(nrm, _f), _p(off, _f)))
        return near, nrm, off


def ref_pcg(row_start, col_index, blocks, pinned, active, normals, grad, max_iterations=50, tolerance=1e-2):
    L = ref()
    n = len(row_start) - 1
    rs, ci = _np(row_start, np.uint32), _np(col_index, np.uint32)
    bl = _np(blocks, np.float32).reshape(-1, 9)
    pn, ac = _np(pinned, np.uint8), _np(active, np.uint8)
    nm, g = _np(normals, np.float32), _np(grad, np.float32)
    step, resid, its = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), C.c_int()
    code = L.ref_pcg(n, _p(rs, _u32), _p(ci, _u32), _p(bl, _f), _p(pn, _u8), _p(ac, _u8), _p(nm, _f), _p(g, _f),
                     max_iterations, tolerance, _p(step, _f), _p(resid, _f), C.byref(its))
    _raise(code, "ref_pcg failed")
    return step, resid, its.value
