"""Pattern -> simulation mesh (include/drape_mesh.h, host code): the reference's sim-mesh tests
(libs/garment/tests/test_sim_mesh.cpp) restated on rectangles, a disc and sewn rectangles (the reference's test tee
generator is outside this build), plus a mesh driving the solver's model build. The reference's CDT library is absent,
so the triangulation itself is pinned by these properties, not by the library's output."""
import ctypes as C
import math

import numpy as np
import pytest

from drape_b200 import mesher as M
from drape_b200.scene import Scene, SceneDesc, drape_scene_desc, jersey_fabric


def tri_areas(m):
    a = m.rest[m.triangles]
    return 0.5 * ((a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1]) - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0]))


def min_angle_deg(m):
    p = m.rest[m.triangles]
    worst = 180.0
    for k in range(3):
        a = p[:, (k + 1) % 3] - p[:, k]
        b = p[:, (k + 2) % 3] - p[:, k]
        c = np.sum(a * b, axis=1) / (np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1))
        worst = min(worst, float(np.degrees(np.arccos(np.clip(c, -1, 1))).min()))
    return worst


def single(piece):
    return M.Pattern([piece])


def two_rects_sewn():
    a, b = M.rectangle_piece("sq1", 0.2, 0.1), M.rectangle_piece("sq2", 0.2, 0.1)
    return M.Pattern([a, b], [M.SeamSpec("s1", M.segment_edge(a, "right", "right", False),
                                         M.segment_edge(b, "left", "left", True))])


def test_particle_distances():
    """test_sim_mesh.cpp ParticleDistances."""
    assert M.particle_distance("draft") == 0.020
    assert M.particle_distance("standard") == 0.010
    assert M.particle_distance("fine") == 0.005


def test_seam_pairs_are_one_to_one():
    """test_sim_mesh.cpp SeamPairsAreOneToOne: 11 pairs at 1 cm on a 0.1 m seam, in order, across the pieces."""
    m = M.build_sim_mesh(two_rects_sewn(), 0.01)
    assert len(m.seam_pairs) == 11
    for i, (a, b, seam, index) in enumerate(m.seam_pairs):
        assert index == i and seam == 0
        assert m.vertex_piece[a] == 0 and m.vertex_piece[b] == 1
        assert abs(m.rest[a, 1] - m.rest[b, 1]) < 1e-9
        assert abs(m.rest[a, 0] - 0.2) < 1e-12 and abs(m.rest[b, 0]) < 1e-12


def test_area_is_preserved():
    """test_sim_mesh.cpp AreaIsPreserved."""
    m = M.build_sim_mesh(single(M.rectangle_piece("r", 0.2, 0.1)), 0.01)
    assert abs(tri_areas(m).sum() - 0.02) < 1e-9


@pytest.mark.parametrize("h", [0.02, 0.01, 0.005])
def test_vertex_area_sums_to_total(h):
    """test_sim_mesh.cpp VertexAreaSumsToTotal (two sewn rectangles and a disc in place of the test tee)."""
    pat = two_rects_sewn()
    pat.pieces.append(M.disc_piece(0.08, "disc"))
    m = M.build_sim_mesh(pat, h)
    assert abs(m.vertex_area.sum() - tri_areas(m).sum()) < 1e-12
    assert len(m.vertex_area) == len(m.rest) == len(m.boundary) == len(m.vertex_piece)
    assert len(m.triangle_piece) == len(m.triangles)
    assert len(m.piece_grain) == 3
    # The disc's outline is sampled with chords ~h long (area deficit ~ perimeter h^2 / 12 r) of cubic arcs.
    assert abs(tri_areas(m).sum() - (0.04 + math.pi * 0.08 ** 2)) < 5e-5 + 0.6 * h * h


def test_triangles_are_well_shaped():
    """test_sim_mesh.cpp TrianglesAreWellShaped: minimum angle >= 15 degrees, every triangle counter-clockwise."""
    assert min_angle_deg(M.build_sim_mesh(single(M.rectangle_piece("r", 0.2, 0.1)), 0.01)) >= 15.0
    assert min_angle_deg(M.build_sim_mesh(single(M.disc_piece(0.1)), 0.01)) >= 15.0
    for h in (0.020, 0.010, 0.005):
        pat = two_rects_sewn()
        pat.pieces.append(M.disc_piece(0.1, "disc"))
        m = M.build_sim_mesh(pat, h)
        assert min_angle_deg(m) >= 15.0, h
        assert (tri_areas(m) > 0).all()


@pytest.mark.parametrize("grain_deg", [0.0, 30.0])
def test_lattice_follows_grain(grain_deg):
    """test_sim_mesh.cpp LatticeFollowsGrain: >= 80 % of interior edges within 2 degrees of the grain's 60-degree
    directions."""
    g = math.radians(grain_deg)
    m = M.build_sim_mesh(single(M.rectangle_piece("r", 0.3, 0.3, (math.cos(g), math.sin(g)))), 0.01)
    edges = set()
    for t in m.triangles:
        for k in range(3):
            a, b = int(t[k]), int(t[(k + 1) % 3])
            if m.boundary[a] or m.boundary[b]:
                continue
            edges.add((min(a, b), max(a, b)))
    aligned = 0
    for a, b in edges:
        d = m.rest[b] - m.rest[a]
        ang = math.degrees(math.atan2(d[1], d[0])) - grain_deg
        ang = math.fmod(math.fmod(ang, 60.0) + 60.0, 60.0)
        aligned += min(ang, 60.0 - ang) <= 2.0
    assert aligned >= 0.8 * len(edges)


def test_corners_are_vertices():
    """test_sim_mesh.cpp CornersAreVertices: every outline corner (> 10 degrees) is a mesh vertex."""
    pat = two_rects_sewn()
    m = M.build_sim_mesh(pat, 0.02)
    for pi, piece in enumerate(pat.pieces):
        for _, seg in piece.segments:
            p0 = np.asarray(seg)[0]
            on = (m.vertex_piece == pi) & (np.linalg.norm(m.rest - p0, axis=1) < 1e-12)
            assert on.any(), (piece.id, p0)


def test_thin_piece_is_valid():
    """test_sim_mesh.cpp ThinPieceIsValid."""
    m = M.build_sim_mesh(single(M.rectangle_piece("thin", 0.5, 0.02)), 0.02)
    assert len(m.triangles) > 0
    assert (tri_areas(m) > 1e-12).all()
    assert np.isfinite(m.rest).all()


def test_invalid_pattern_raises():
    """test_sim_mesh.cpp InvalidPatternThrows: an open outline names the rule "outline-closed"."""
    p = M.rectangle_piece("open", 0.1, 0.1)
    p.segments = p.segments[:-1]
    with pytest.raises(M.MeshError, match="outline-closed"):
        M.build_sim_mesh(single(p), 0.01)


@pytest.mark.parametrize("mutate,rule", [
    (lambda pat: setattr(pat.seams[0].b, "reversed", False), "seam-twisted"),
    (lambda pat: setattr(pat.seams[0].a, "end", 5.0), "seam-range"),
    (lambda pat: setattr(pat.seams[0].b, "piece", "nope"), "seam-piece"),
    (lambda pat: setattr(pat.seams[0].a, "start", 0.25), "seam-length"),
    (lambda pat: setattr(pat.pieces[0], "grain", (0.0, 0.0)), "grainline"),
    (lambda pat: setattr(pat.pieces[0], "fabric_slot", ""), "fabric-slot"),
])
def test_validation_rules(mutate, rule):
    """validate.cpp:25-87: each broken rule is named in the error."""
    pat = two_rects_sewn()
    mutate(pat)
    with pytest.raises(M.MeshError, match=rule):
        M.build_sim_mesh(pat, 0.01)


def test_clockwise_outline_is_rejected():
    p = M.rectangle_piece("cw", 0.1, 0.1)
    p.segments = [(n, np.asarray(s)[::-1]) for n, s in reversed(p.segments)]
    with pytest.raises(M.MeshError, match="outline-ccw"):
        M.build_sim_mesh(single(p), 0.01)


def test_mesh_drives_the_solver_model(cuda_mod):
    """The mesh's arrays are a garment: the solver's host model builds from it (structure, seams and hinges)."""
    m = M.build_sim_mesh(two_rects_sewn(), 0.01)
    g = M.to_garment(m, "pair", [jersey_fabric(), jersey_fabric()])
    desc = SceneDesc(Scene([g]))
    L = cuda_mod.load()
    L.drape_model_build.argtypes = [C.POINTER(drape_scene_desc), C.POINTER(C.c_void_p)]
    L.drape_model_structure_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_uint32)]
    L.drape_model_destroy.argtypes = [C.c_void_p]
    h = C.c_void_p()
    assert L.drape_model_build(desc.ptr(), C.byref(h)) == 0
    try:
        sz = (C.c_uint32 * 5)()
        assert L.drape_model_structure_sizes(h, sz) == 0
        n, B, S, H, K = list(sz)
        assert n == len(m.rest) and S == len(m.triangles) and K == len(m.seam_pairs)
        assert H > 0 and B > n
    finally:
        L.drape_model_destroy(h)


def _polygon_piece(pid, pts, grain=(0.0, 1.0)):
    pts = [np.asarray(p, np.float64) for p in pts]
    return M.Piece(pid, [(f"e{i}", M.line(pts[i], pts[(i + 1) % len(pts)])) for i in range(len(pts))], grain, "body")


@pytest.mark.parametrize("h", [0.02, 0.01, 0.005])
def test_concave_piece_keeps_its_notch(h):
    """An L-shaped piece: the triangulation covers the outline exactly (area to 1e-9) and no triangle crosses the
    notch (every centroid lies inside the L), so the outline constraint and the removal of the outside hold."""
    pts = [(0, 0), (0.3, 0), (0.3, 0.1), (0.1, 0.1), (0.1, 0.3), (0, 0.3)]
    m = M.build_sim_mesh(single(_polygon_piece("L", pts, (0.6, 0.8))), h)
    assert abs(tri_areas(m).sum() - (0.3 * 0.1 + 0.1 * 0.2)) < 1e-9
    c = m.rest[m.triangles].mean(axis=1)
    inside = ((c[:, 0] <= 0.3) & (c[:, 1] <= 0.1)) | ((c[:, 0] <= 0.1) & (c[:, 1] <= 0.3))
    assert inside.all() and (c >= 0).all()
    assert (tri_areas(m) > 0).all() and min_angle_deg(m) >= 15.0


def test_every_outline_edge_is_a_mesh_edge():
    """The outline samples, in order, are joined by mesh edges (the constraint edges of the triangulation)."""
    pat = two_rects_sewn()
    pat.pieces.append(M.disc_piece(0.07, "disc"))
    m = M.build_sim_mesh(pat, 0.01)
    edges = set()
    for t in m.triangles:
        for k in range(3):
            a, b = int(t[k]), int(t[(k + 1) % 3])
            edges.add((min(a, b), max(a, b)))
    for pi in range(len(pat.pieces)):
        idx = np.nonzero((m.vertex_piece == pi) & (m.boundary == 1))[0]
        # Boundary vertices come first in each piece, in outline order.
        assert np.array_equal(idx, np.arange(idx[0], idx[0] + len(idx)))
        for k in range(len(idx)):
            a, b = int(idx[k]), int(idx[(k + 1) % len(idx)])
            assert (min(a, b), max(a, b)) in edges, (pi, k)
