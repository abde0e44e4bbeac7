"""ctypes binding of the pattern -> simulation mesh builder (include/drape_mesh.h): buildSimMesh
(libs/garment/src/sim_mesh_builder.cpp:196-323) on the host, plus the pattern helpers the reference's tests use
(rectanglePiece, libs/garment/src/shapes.cpp:5-17; segmentEdge, libs/core/src/pattern.cpp:15-26).

A mesh's arrays are the garment arrays of a solver scene: ``to_garment`` places it flat at a height and returns a
scene.Garment for any Solver.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import cuda as _cuda

_P = C.POINTER


class drape_bezier(C.Structure):
    _fields_ = [("p", C.c_double * 8)]


class drape_piece_desc(C.Structure):
    _fields_ = [("id", C.c_char_p), ("segments", _P(drape_bezier)), ("segment_count", C.c_uint32),
                ("grain", C.c_double * 2), ("fabric_slot", C.c_char_p)]


class drape_seam_desc(C.Structure):
    _fields_ = [("id", C.c_char_p), ("piece_a", C.c_char_p), ("start_a", C.c_double), ("end_a", C.c_double),
                ("reversed_a", C.c_int32), ("piece_b", C.c_char_p), ("start_b", C.c_double), ("end_b", C.c_double),
                ("reversed_b", C.c_int32), ("ease", C.c_double)]


class drape_pattern_desc(C.Structure):
    _fields_ = [("pieces", _P(drape_piece_desc)), ("piece_count", C.c_uint32), ("seams", _P(drape_seam_desc)),
                ("seam_count", C.c_uint32)]


class MeshError(ValueError):
    """An invalid pattern (the message lists the validation rule ids), as the reference's MeshError."""


def _lib():
    L = _cuda.load()
    if getattr(L, "_mesh_bound", False):
        return L
    L.drape_mesh_particle_distance.restype = C.c_double
    L.drape_mesh_particle_distance.argtypes = [C.c_int]
    L.drape_mesh_build.argtypes = [_P(drape_pattern_desc), C.c_double, _P(C.c_void_p)]
    L.drape_mesh_destroy.argtypes = [C.c_void_p]
    L.drape_mesh_last_error.restype = C.c_char_p
    L.drape_mesh_sizes.argtypes = [C.c_void_p, _P(C.c_uint32)]
    L.drape_mesh_read.argtypes = [C.c_void_p, _P(C.c_double), _P(C.c_uint32), _P(C.c_uint8), _P(C.c_double),
                                  _P(C.c_uint32), _P(C.c_uint32), _P(C.c_double), _P(C.c_uint32)]
    L._mesh_bound = True
    return L


def particle_distance(quality: str) -> float:
    """particleDistance (sim_mesh_builder.cpp:14-21): Draft 0.020, Standard 0.010, Fine 0.005 m."""
    return _lib().drape_mesh_particle_distance({"draft": 0, "standard": 1, "fine": 2}[quality.lower()])


# ---- pattern ----

_GX = np.array([-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640])
_GW = np.array([0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665, 0.2369268850561891])


def bezier_length(p: np.ndarray, intervals: int = 256) -> float:
    """Arc length of a cubic segment (4 x 2 control points) with the mesher's table: 256 intervals, 5-point
    Gauss-Legendre quadrature of the speed in each (libs/core/src/bezier.cpp:29-59)."""
    a = np.arange(intervals) / intervals
    half = 0.5 / intervals
    t = (a + half)[:, None] + half * _GX[None, :]
    u = 1.0 - t
    d = (3 * u * u)[..., None] * (p[1] - p[0]) + (6 * u * t)[..., None] * (p[2] - p[1]) + \
        (3 * t * t)[..., None] * (p[3] - p[2])
    speed = np.linalg.norm(d, axis=-1)
    return float(np.sum((speed * _GW[None, :]).sum(axis=1) * half))


def line(a, b) -> np.ndarray:
    """CubicBezier::line (bezier.cpp:25-27): control points at thirds."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.stack([a, a + (b - a) / 3.0, a + 2.0 * (b - a) / 3.0, b])


@dataclass
class Piece:
    id: str
    segments: List[Tuple[str, np.ndarray]]  # (name, 4 x 2 control points), counter-clockwise
    grain: Tuple[float, float] = (0.0, 1.0)
    fabric_slot: str = "body"

    def segment_starts(self) -> np.ndarray:
        lengths = [bezier_length(np.asarray(s, np.float64)) for _, s in self.segments]
        return np.concatenate([[0.0], np.cumsum(lengths)])

    def perimeter(self) -> float:
        return float(self.segment_starts()[-1])


@dataclass
class EdgeRef:
    piece: str
    start: float
    end: float
    reversed: bool = False


@dataclass
class SeamSpec:
    id: str
    a: EdgeRef
    b: EdgeRef
    ease: float = 0.0


@dataclass
class Pattern:
    pieces: List[Piece] = field(default_factory=list)
    seams: List[SeamSpec] = field(default_factory=list)


def rectangle_piece(pid: str, width: float, height: float, grain=(0.0, 1.0), fabric_slot: str = "body") -> Piece:
    """rectanglePiece (shapes.cpp:5-17): bottom, right, top, left."""
    return Piece(pid, [("bottom", line((0, 0), (width, 0))), ("right", line((width, 0), (width, height))),
                       ("top", line((width, height), (0, height))), ("left", line((0, height), (0, 0)))],
                 tuple(grain), fabric_slot)


def disc_piece(r: float, pid: str = "disc") -> Piece:
    """A disc of four cubic quarter arcs centred at (r, r)."""
    k = 0.5522847498 * r
    c = np.array([r, r])
    arcs = [[(r, 0), (r, k), (k, r), (0, r)], [(0, r), (-k, r), (-r, k), (-r, 0)],
            [(-r, 0), (-r, -k), (-k, -r), (0, -r)], [(0, -r), (k, -r), (r, -k), (r, 0)]]
    return Piece(pid, [(f"q{i}", c + np.array(a, np.float64)) for i, a in enumerate(arcs)], (0.0, 1.0), "body")


def segment_edge(piece: Piece, first: str, last: str, reversed_: bool) -> EdgeRef:
    """segmentEdge (pattern.cpp:15-26): the arc-length range from the start of `first` to the end of `last`."""
    names = [n for n, _ in piece.segments]
    i, k = names.index(first), names.index(last)
    if k < i:
        raise ValueError(f"piece '{piece.id}': segment '{last}' comes before '{first}'")
    st = piece.segment_starts()
    return EdgeRef(piece.id, float(st[i]), float(st[k + 1]), reversed_)


# ---- mesh ----

@dataclass
class SimMesh:
    rest: np.ndarray          # (V, 2) pattern-space positions, m
    vertex_piece: np.ndarray  # (V,)
    boundary: np.ndarray      # (V,) 1 on the piece outline
    vertex_area: np.ndarray   # (V,) a third of the incident triangle areas, m^2
    triangles: np.ndarray     # (T, 3) counter-clockwise
    triangle_piece: np.ndarray
    piece_grain: np.ndarray   # (P, 2) unit grainlines
    seam_pairs: np.ndarray    # (K, 4) a, b, seam, index


class _PatternDesc:
    def __init__(self, pattern: Pattern):
        self._keep = []
        pieces = (drape_piece_desc * max(1, len(pattern.pieces)))()
        for i, p in enumerate(pattern.pieces):
            segs = (drape_bezier * max(1, len(p.segments)))()
            for k, (_, cp) in enumerate(p.segments):
                segs[k].p[:] = [float(v) for v in np.asarray(cp, np.float64).reshape(-1)]
            pid, slot = p.id.encode(), p.fabric_slot.encode()
            self._keep += [segs, pid, slot]
            pieces[i] = drape_piece_desc(pid, C.cast(segs, _P(drape_bezier)), len(p.segments),
                                         (C.c_double * 2)(*p.grain), slot)
        seams = (drape_seam_desc * max(1, len(pattern.seams)))()
        for i, s in enumerate(pattern.seams):
            sid, pa, pb = s.id.encode(), s.a.piece.encode(), s.b.piece.encode()
            self._keep += [sid, pa, pb]
            seams[i] = drape_seam_desc(sid, pa, s.a.start, s.a.end, int(s.a.reversed), pb, s.b.start, s.b.end,
                                       int(s.b.reversed), s.ease)
        self._keep += [pieces, seams]
        self.desc = drape_pattern_desc(C.cast(pieces, _P(drape_piece_desc)), len(pattern.pieces),
                                       C.cast(seams, _P(drape_seam_desc)), len(pattern.seams))


def build_sim_mesh(pattern: Pattern, h: float) -> SimMesh:
    """buildSimMesh(pattern, particleDistance) (sim_mesh_builder.hpp:19); raises MeshError for an invalid pattern."""
    L = _lib()
    pd = _PatternDesc(pattern)
    handle = C.c_void_p()
    code = L.drape_mesh_build(C.byref(pd.desc), float(h), C.byref(handle))
    if code != 0:
        msg = L.drape_mesh_last_error().decode()
        raise MeshError(msg) if code == -1 else RuntimeError(msg)
    try:
        sz = (C.c_uint32 * 4)()
        if L.drape_mesh_sizes(handle, sz) != 0:
            raise RuntimeError(L.drape_mesh_last_error().decode())
        V, T, P, K = list(sz)
        m = SimMesh(np.zeros((V, 2)), np.zeros(V, np.uint32), np.zeros(V, np.uint8), np.zeros(V),
                    np.zeros((T, 3), np.uint32), np.zeros(T, np.uint32), np.zeros((P, 2)), np.zeros((K, 4), np.uint32))
        d, u, b = (lambda a: a.ctypes.data_as(_P(C.c_double))), (lambda a: a.ctypes.data_as(_P(C.c_uint32))), \
            (lambda a: a.ctypes.data_as(_P(C.c_uint8)))
        if L.drape_mesh_read(handle, d(m.rest), u(m.vertex_piece), b(m.boundary), d(m.vertex_area), u(m.triangles),
                             u(m.triangle_piece), d(m.piece_grain), u(m.seam_pairs)) != 0:
            raise RuntimeError(L.drape_mesh_last_error().decode())
        return m
    finally:
        L.drape_mesh_destroy(handle)


def to_garment(mesh: SimMesh, gid: str, piece_fabrics: Sequence, height: float = 0.5,
               offsets: Optional[Sequence[Tuple[float, float, float]]] = None):
    """A scene.Garment of the mesh: pattern (x, y) laid flat at z = height (plus a per-piece offset), the pieces'
    fabrics in pattern order."""
    from .scene import Garment
    n = len(mesh.rest)
    x = np.zeros((n, 3))
    x[:, 0], x[:, 1], x[:, 2] = mesh.rest[:, 0], mesh.rest[:, 1], height
    if offsets is not None:
        x += np.asarray(offsets, np.float64)[mesh.vertex_piece]
    return Garment(id=gid, rest=mesh.rest.copy(), vertex_piece=mesh.vertex_piece.astype(np.uint32),
                   vertex_area=mesh.vertex_area.copy(), triangles=mesh.triangles.astype(np.uint32),
                   triangle_piece=mesh.triangle_piece.astype(np.uint32), piece_grain=mesh.piece_grain.copy(),
                   piece_fabric=list(piece_fabrics), seam_pairs=mesh.seam_pairs.astype(np.uint32),
                   initial_positions=x)
