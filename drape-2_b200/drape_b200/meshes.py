"""Closed triangle meshes for collision bodies: the reference's primitives (libs/avatar/src/primitives.cpp: icosphere,
ring-based capsule and elliptic capsule, box), its static test body (libs/avatar/src/test_body.cpp), and the
capsule-union body of the tube workloads as meshes. Built in FP64 in the same construction order as the reference
(vertex order, triangle order, outward orientation by signed volume); used as input to the collision-field bake
(drape_b200.bake) and its tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, List, Sequence

import numpy as np


@dataclass
class TriangleMesh:
    vertices: np.ndarray   # (V, 3) float64
    triangles: np.ndarray  # (T, 3) uint32, counter-clockwise seen from outside


def signed_volume(m: TriangleMesh) -> float:
    """libs/core/src/triangle_mesh.cpp:8-14."""
    v = m.vertices
    t = m.triangles.astype(np.int64)
    return float(np.sum(np.einsum("ij,ij->i", v[t[:, 0]], np.cross(v[t[:, 1]], v[t[:, 2]])))) / 6.0


def _outward(m: TriangleMesh) -> TriangleMesh:
    if signed_volume(m) < 0:
        m.triangles = m.triangles[:, [0, 2, 1]].copy()
    return m


def is_closed_manifold(m: TriangleMesh) -> bool:
    """Every directed edge exactly once, and its reverse exactly once (triangle_mesh.cpp:16-28)."""
    if len(m.triangles) == 0:
        return False
    t = m.triangles.astype(np.int64)
    e = np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [2, 0]]])
    keys = e[:, 0] << 32 | e[:, 1]
    if len(np.unique(keys)) != len(keys):
        return False
    rev = e[:, 1] << 32 | e[:, 0]
    return bool(np.all(np.isin(rev, keys)))


def _ring_surface(south, north, ring_count: int, segments: int, point: Callable[[int, int], np.ndarray]):
    verts = [np.asarray(south, dtype=np.float64)]
    for r in range(ring_count):
        for s in range(segments):
            verts.append(point(r, s))
    verts.append(np.asarray(north, dtype=np.float64))
    north_idx = len(verts) - 1

    def idx(r, s):
        return 1 + r * segments + (s % segments)

    tris = [(0, idx(0, s + 1), idx(0, s)) for s in range(segments)]
    for r in range(ring_count - 1):
        for s in range(segments):
            tris.append((idx(r, s), idx(r, s + 1), idx(r + 1, s + 1)))
            tris.append((idx(r, s), idx(r + 1, s + 1), idx(r + 1, s)))
    tris += [(north_idx, idx(ring_count - 1, s), idx(ring_count - 1, s + 1)) for s in range(segments)]
    return _outward(TriangleMesh(np.asarray(verts), np.asarray(tris, dtype=np.uint32)))


def _ring_latitude(r: int, rings: int) -> float:
    """Ring latitudes of a capsule with `rings` rings per hemisphere; the equator appears twice."""
    if r < rings:
        return -math.pi / 2 + (r + 1) * (math.pi / 2) / rings
    return (r - rings) * (math.pi / 2) / rings


def _normalized(v):
    v = np.asarray(v, dtype=np.float64)
    n = math.sqrt(float(v @ v))
    return v / n if n > 0 else v


def icosphere(center, radius: float, subdivisions: int) -> TriangleMesh:
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [_normalized(p) for p in ((-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
                                  (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1))]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        mid = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                v.append(_normalized(v[a] + v[b]))
                mid[key] = len(v) - 1
            return mid[key]

        nxt = []
        for tri in f:
            a, b, c = midpoint(tri[0], tri[1]), midpoint(tri[1], tri[2]), midpoint(tri[2], tri[0])
            nxt += [(tri[0], a, c), (tri[1], b, a), (tri[2], c, b), (a, b, c)]
        f = nxt
    c = np.asarray(center, dtype=np.float64)
    return _outward(TriangleMesh(np.asarray([c + radius * p for p in v]), np.asarray(f, dtype=np.uint32)))


def capsule(a, b, radius: float, segments: int = 32, rings: int = 8) -> TriangleMesh:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    w = _normalized(b - a)
    u = np.cross(w, (1.0, 0.0, 0.0)) if abs(w[0]) < 0.9 else np.cross(w, (0.0, 1.0, 0.0))
    u = _normalized(u)
    v = np.cross(w, u)

    def point(r, s):
        phi = _ring_latitude(r, rings)
        lam = 2 * math.pi * s / segments
        c = a if r < rings else b
        return c + radius * (math.cos(phi) * (math.cos(lam) * u + math.sin(lam) * v) + math.sin(phi) * w)

    return _ring_surface(a - radius * w, b + radius * w, 2 * rings, segments, point)


def elliptic_capsule(y_bottom: float, y_top: float, rx: float, rz: float, cap_height: float, segments: int = 48,
                     rings: int = 12) -> TriangleMesh:
    def point(r, s):
        phi = _ring_latitude(r, rings)
        lam = 2 * math.pi * s / segments
        y = (y_bottom if r < rings else y_top) + cap_height * math.sin(phi)
        return np.array([rx * math.cos(phi) * math.cos(lam), y, rz * math.cos(phi) * math.sin(lam)])

    return _ring_surface((0.0, y_bottom - cap_height, 0.0), (0.0, y_top + cap_height, 0.0), 2 * rings, segments,
                         point)


def box(center, half, rotation=np.eye(3)) -> TriangleMesh:
    c, h, R = (np.asarray(x, dtype=np.float64) for x in (center, half, rotation))
    verts = [c + R @ np.array([(1 if i & 1 else -1) * h[0], (1 if i & 2 else -1) * h[1], (1 if i & 4 else -1) * h[2]])
             for i in range(8)]
    tris = [(0, 2, 3), (0, 3, 1), (4, 5, 7), (4, 7, 6), (0, 1, 5), (0, 5, 4), (2, 6, 7), (2, 7, 3), (0, 4, 6),
            (0, 6, 2), (1, 3, 7), (1, 7, 5)]
    return _outward(TriangleMesh(np.asarray(verts), np.asarray(tris, dtype=np.uint32)))


def test_body() -> List[TriangleMesh]:
    """The reference's static test body (test_body.cpp:9-29): torso, neck, head and A-pose arms."""
    s = math.sqrt(0.5)
    dl, dr = np.array([s, -s, 0.0]), np.array([-s, -s, 0.0])
    sl, sr = np.array([0.19, 1.37, 0.0]), np.array([-0.19, 1.37, 0.0])
    return [elliptic_capsule(0.85, 1.38, 0.17, 0.11, 0.08), capsule((0, 1.40, 0), (0, 1.58, 0), 0.055),
            icosphere((0, 1.68, 0), 0.10, 3), capsule(sl, sl + 0.55 * dl, 0.045), capsule(sr, sr + 0.55 * dr, 0.045)]


def capsule_union_body(torso_radius: float = 0.15, arm_radius: float = 0.05, torso_half: float = 0.3,
                       arm_length: float = 0.45, segments: int = 48, rings: int = 12) -> List[TriangleMesh]:
    """The tube workloads' body (drape_b200.scenes.capsule_union_sdf) as three closed capsule meshes: the torso along
    z through the origin, and two arms leaving its end points outward along +-z at 45 degrees below horizontal."""
    c, s = math.cos(math.radians(45.0)), math.sin(math.radians(45.0))
    parts = [capsule((0.0, 0.0, -torso_half), (0.0, 0.0, torso_half), torso_radius, segments, rings)]
    for sign in (1.0, -1.0):
        root = np.array([0.0, 0.0, sign * torso_half])
        tip = np.array([0.0, -arm_length * s, sign * (torso_half + arm_length * c)])
        parts.append(capsule(root, tip, arm_radius, segments // 2, rings // 2))
    return parts


def triangle_count(components: Sequence[TriangleMesh]) -> int:
    return int(sum(len(m.triangles) for m in components))
