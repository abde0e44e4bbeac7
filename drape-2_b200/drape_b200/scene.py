"""Scene description on the host: numpy arrays plus their ctypes view as ``drape_scene_desc`` (include/drape_scene.h).

The dataclasses restate the reference's scene types with numpy arrays in place of Eigen vectors:
``Fabric`` <- drape::FabricPhysical (libs/core/include/drape/core/fabric.hpp:10-18), ``Garment`` <- SimGarment + SimMesh
(libs/sim/include/drape/sim/solver.hpp:32-37, libs/core/include/drape/core/sim_mesh.hpp:14-30), ``Field`` <-
CollisionField (libs/core/include/drape/core/collision_field.hpp:11-20), ``Settings`` <- SimSettings (solver.hpp:19-30),
``Scene`` <- SimScene (solver.hpp:49-55).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np


class drape_fabric(C.Structure):
    _fields_ = [(name, C.c_double) for name in (
        "stretch_warp", "stretch_weft", "stretch_bias", "strain_limit_warp", "strain_limit_weft",
        "bend_warp", "bend_weft", "weight", "thickness", "friction", "damping")]


class drape_garment_desc(C.Structure):
    _fields_ = [
        ("id", C.c_char_p),
        ("vertex_count", C.c_uint32),
        ("rest", C.POINTER(C.c_double)),
        ("vertex_piece", C.POINTER(C.c_uint32)),
        ("vertex_area", C.POINTER(C.c_double)),
        ("triangle_count", C.c_uint32),
        ("triangles", C.POINTER(C.c_uint32)),
        ("triangle_piece", C.POINTER(C.c_uint32)),
        ("piece_count", C.c_uint32),
        ("piece_grain", C.POINTER(C.c_double)),
        ("piece_fabric", C.POINTER(drape_fabric)),
        ("seam_pair_count", C.c_uint32),
        ("seam_pairs", C.POINTER(C.c_uint32)),
        ("initial_positions", C.POINTER(C.c_double)),
    ]


class drape_field_desc(C.Structure):
    _fields_ = [
        ("origin", C.c_double * 3),
        ("cell_size", C.c_double),
        ("dims", C.c_int32 * 3),
        ("band", C.c_double),
        ("values", C.POINTER(C.c_float)),
    ]


class drape_settings(C.Structure):
    _fields_ = [
        ("gravity", C.c_double * 3),
        ("collision_offset", C.c_double),
        ("assembly_closing_speed", C.c_double),
        ("assembly_extra_damping", C.c_double),
        ("damping_scale", C.c_double),
        ("strain_limit_stiffness_scale", C.c_double),
        ("seam_stiffness", C.c_double),
        ("friction_slip_speed", C.c_double),
        ("max_cg_iterations", C.c_int32),
        ("cg_tolerance", C.c_double),
    ]


class drape_scene_desc(C.Structure):
    _fields_ = [
        ("garment_count", C.c_uint32),
        ("garments", C.POINTER(drape_garment_desc)),
        ("body", C.POINTER(drape_field_desc)),
        ("pin_count", C.c_uint32),
        ("pin_particles", C.POINTER(C.c_uint32)),
        ("pin_positions", C.POINTER(C.c_double)),
        ("force_count", C.c_uint32),
        ("force_particles", C.POINTER(C.c_uint32)),
        ("forces", C.POINTER(C.c_double)),
        ("settings", drape_settings),
    ]


class drape_stats(C.Structure):
    _fields_ = [
        ("has_non_finite", C.c_int32),
        ("kinetic_energy", C.c_double),
        ("rms_speed", C.c_double),
        ("max_seam_gap", C.c_double),
        ("max_body_penetration", C.c_double),
    ]


class drape_counters(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "substeps", "newton_iterations", "cg_iterations", "line_search_halvings", "precond_fallbacks",
        "learned_solves", "pcg_nanoseconds")]


class drape_drape_options(C.Structure):
    _fields_ = [
        ("substeps", C.c_int32),
        ("iterations", C.c_int32),
        ("frame_dt", C.c_double),
        ("max_assembly_seconds", C.c_double),
        ("seam_gap_done", C.c_double),
        ("settle_rms_speed", C.c_double),
        ("settle_hold_frames", C.c_int32),
        ("max_sim_seconds", C.c_double),
        ("snapshot_every", C.c_int32),
        ("max_retries", C.c_int32),
        ("energy_rise_frames", C.c_int32),
        ("frames_per_wait", C.c_int32),
    ]


class drape_drape_result(C.Structure):
    _fields_ = [
        ("settled", C.c_int32),
        ("failed", C.c_int32),
        ("simulated_seconds", C.c_double),
        ("retries", C.c_int32),
        ("frames_run", C.c_int32),
        ("assembly_end_seam_gap", C.c_double),
        ("assembly_seconds", C.c_double),
    ]


ASSEMBLING, SETTLING = 0, 1


@dataclass
class Fabric:
    """FabricPhysical in SI units."""
    stretch_warp: float = 0.0
    stretch_weft: float = 0.0
    stretch_bias: float = 0.0
    strain_limit_warp: float = 0.0
    strain_limit_weft: float = 0.0
    bend_warp: float = 0.0
    bend_weft: float = 0.0
    weight: float = 0.0
    thickness: float = 0.0
    friction: float = 0.0
    damping: float = 0.0

    def to_c(self) -> drape_fabric:
        return drape_fabric(*[float(getattr(self, f[0])) for f in drape_fabric._fields_])


def jersey_fabric() -> Fabric:
    """The reference's jersey test fabric (libs/core/src/test_fabrics.cpp:5)."""
    return Fabric(400, 200, 100, 0.5, 0.8, 2e-6, 1.5e-6, 0.160, 0.0006, 0.3, 0.3)


def stiff_fabric() -> Fabric:
    """libs/core/src/test_fabrics.cpp:7."""
    return Fabric(20000, 20000, 5000, 0.02, 0.02, 100e-6, 100e-6, 0.450, 0.0008, 0.3, 1.0)


@dataclass
class Garment:
    id: str
    rest: np.ndarray                # (V, 2) float64
    vertex_piece: np.ndarray        # (V,) uint32
    vertex_area: np.ndarray         # (V,) float64
    triangles: np.ndarray           # (T, 3) uint32, CCW in pattern space
    triangle_piece: np.ndarray      # (T,) uint32
    piece_grain: np.ndarray         # (P, 2) float64
    piece_fabric: List[Fabric]
    seam_pairs: np.ndarray          # (Q, 4) uint32: a, b, seam, index
    initial_positions: np.ndarray   # (V, 3) float64
    boundary: Optional[np.ndarray] = None

    @property
    def vertex_count(self) -> int:
        return int(self.rest.shape[0])


@dataclass
class Field:
    origin: np.ndarray
    cell_size: float
    dims: tuple
    band: float
    values: np.ndarray  # float32, shape (dz, dy, dx) -> x fastest when flattened

    def sample(self, p: np.ndarray) -> np.ndarray:
        """Trilinear sample in float64 (collision_field.cpp:8-30), vectorised over rows of p."""
        p = np.atleast_2d(np.asarray(p, dtype=np.float64))
        local = (p - self.origin) / self.cell_size
        dims = np.asarray(self.dims)
        inside = np.all((local >= 0.0) & (local <= dims - 1), axis=1)
        out = np.full(p.shape[0], self.band, dtype=np.float64)
        if not inside.any():
            return out
        loc = local[inside]
        i = np.minimum(np.floor(loc).astype(np.int64), dims - 2)
        t = loc - i
        v = self.values.reshape(-1)
        acc = np.zeros(loc.shape[0])
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    w = ((t[:, 0] if dx else 1 - t[:, 0]) * (t[:, 1] if dy else 1 - t[:, 1]) *
                         (t[:, 2] if dz else 1 - t[:, 2]))
                    idx = ((i[:, 2] + dz) * dims[1] + (i[:, 1] + dy)) * dims[0] + (i[:, 0] + dx)
                    acc += w * v[idx].astype(np.float64)
        out[inside] = acc
        return out


@dataclass
class Settings:
    gravity: tuple = (0.0, -9.81, 0.0)
    collision_offset: float = 0.003
    assembly_closing_speed: float = 0.25
    assembly_extra_damping: float = 10.0
    damping_scale: float = 5.0
    strain_limit_stiffness_scale: float = 100.0
    seam_stiffness: float = 1e4
    friction_slip_speed: float = 3e-4
    max_cg_iterations: int = 50
    cg_tolerance: float = 1e-2

    def to_c(self) -> drape_settings:
        s = drape_settings()
        s.gravity[:] = [float(g) for g in self.gravity]
        for name, _ in drape_settings._fields_[1:]:
            setattr(s, name, getattr(self, name))
        return s


@dataclass
class Scene:
    garments: List[Garment] = field(default_factory=list)
    body: Optional[Field] = None
    pins: List[tuple] = field(default_factory=list)     # (particle, (x, y, z))
    forces: List[tuple] = field(default_factory=list)   # (particle, (fx, fy, fz))
    settings: Settings = field(default_factory=Settings)

    @property
    def particle_count(self) -> int:
        return sum(g.vertex_count for g in self.garments)

    def initial_positions(self) -> np.ndarray:
        x = np.concatenate([g.initial_positions for g in self.garments]) if self.garments else np.zeros((0, 3))
        x = x.copy()
        for p, pos in self.pins:
            x[p] = pos
        return x


def _ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None and a.size else C.POINTER(ctype)()


class SceneDesc:
    """Owns contiguous copies of a Scene's arrays and the drape_scene_desc that points at them."""

    def __init__(self, scene: Scene):
        self._keep = []
        gds = (drape_garment_desc * max(1, len(scene.garments)))()
        for k, g in enumerate(scene.garments):
            rest = self._hold(g.rest, np.float64)
            vp = self._hold(g.vertex_piece, np.uint32)
            va = self._hold(g.vertex_area, np.float64)
            tris = self._hold(g.triangles, np.uint32)
            tp = self._hold(g.triangle_piece, np.uint32)
            grain = self._hold(g.piece_grain, np.float64)
            fabs = (drape_fabric * max(1, len(g.piece_fabric)))(*[f.to_c() for f in g.piece_fabric])
            self._keep.append(fabs)
            sp = self._hold(g.seam_pairs.reshape(-1, 4) if g.seam_pairs is not None else np.zeros((0, 4)), np.uint32)
            init = self._hold(g.initial_positions, np.float64)
            gid = g.id.encode()
            self._keep.append(gid)
            gds[k] = drape_garment_desc(
                gid, g.vertex_count, _ptr(rest, C.c_double), _ptr(vp, C.c_uint32), _ptr(va, C.c_double),
                int(tris.shape[0]), _ptr(tris, C.c_uint32), _ptr(tp, C.c_uint32), int(grain.shape[0]),
                _ptr(grain, C.c_double), C.cast(fabs, C.POINTER(drape_fabric)), int(sp.shape[0]),
                _ptr(sp, C.c_uint32), _ptr(init, C.c_double))
        self._keep.append(gds)
        self.field = None
        body_ptr = C.POINTER(drape_field_desc)()
        if scene.body is not None:
            vals = self._hold(scene.body.values.reshape(-1), np.float32)
            fd = drape_field_desc()
            fd.origin[:] = [float(v) for v in scene.body.origin]
            fd.cell_size = float(scene.body.cell_size)
            fd.dims[:] = [int(d) for d in scene.body.dims]
            fd.band = float(scene.body.band)
            fd.values = _ptr(vals, C.c_float)
            self.field = fd
            body_ptr = C.pointer(fd)
        pin_p = self._hold(np.array([p for p, _ in scene.pins], dtype=np.uint32), np.uint32)
        pin_x = self._hold(np.array([pos for _, pos in scene.pins], dtype=np.float64).reshape(-1, 3), np.float64)
        f_p = self._hold(np.array([p for p, _ in scene.forces], dtype=np.uint32), np.uint32)
        f_f = self._hold(np.array([f for _, f in scene.forces], dtype=np.float64).reshape(-1, 3), np.float64)
        self.desc = drape_scene_desc(
            len(scene.garments), C.cast(gds, C.POINTER(drape_garment_desc)), body_ptr,
            len(scene.pins), _ptr(pin_p, C.c_uint32), _ptr(pin_x, C.c_double),
            len(scene.forces), _ptr(f_p, C.c_uint32), _ptr(f_f, C.c_double), scene.settings.to_c())

    def _hold(self, a, dtype):
        arr = np.ascontiguousarray(np.asarray(a, dtype=dtype))
        self._keep.append(arr)
        return arr

    def ptr(self):
        return C.byref(self.desc)


def field_desc(f: Field):
    """A standalone drape_field_desc for a Field (the caller keeps the returned tuple alive)."""
    vals = np.ascontiguousarray(f.values.reshape(-1), dtype=np.float32)
    fd = drape_field_desc()
    fd.origin[:] = [float(v) for v in f.origin]
    fd.cell_size = float(f.cell_size)
    fd.dims[:] = [int(d) for d in f.dims]
    fd.band = float(f.band)
    fd.values = vals.ctypes.data_as(C.POINTER(C.c_float))
    return fd, vals
