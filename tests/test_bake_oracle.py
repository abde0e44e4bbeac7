"""The collision-field bake's CPU side: the body meshes (the reference's primitives, libs/avatar/tests/
test_primitives.cpp) and the oracle's restatement of bakeCollisionField pinned by the reference's own field tests
(libs/avatar/tests/test_collision_field.cpp, test_collision_perf.cpp)."""
import math
import time

import numpy as np
import pytest

from drape_b200 import meshes as M


def _gradient(field, p):
    """CollisionField::gradient (libs/core/src/collision_field.cpp:32-41): central differences at the cell size."""
    g = np.zeros(3)
    for a in range(3):
        d = np.zeros(3)
        d[a] = field.cell_size
        g[a] = (field.sample(p + d)[0] - field.sample(p - d)[0]) / (2 * field.cell_size)
    n = np.linalg.norm(g)
    return np.zeros(3) if n < 1e-9 else g / n


def _directions(seed, count):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((count, 3))
    return d / np.linalg.norm(d, axis=1)[:, None], rng


def test_primitives_are_closed_and_outward():
    for m in (M.icosphere((0, 0, 0), 0.1, 3), M.capsule((0, 0, 0), (0, 0.3, 0.1), 0.05),
              M.elliptic_capsule(0.85, 1.38, 0.17, 0.11, 0.08), M.box((0.1, 0.2, 0.3), (0.5, 0.05, 0.25))):
        assert M.is_closed_manifold(m)
        assert M.signed_volume(m) > 0


def test_open_mesh_is_not_closed():
    m = M.icosphere((0, 0, 0), 0.1, 1)
    m.triangles = m.triangles[:-1]
    assert not M.is_closed_manifold(m)


def test_volumes_match_analytic():
    r = 0.1
    assert abs(M.signed_volume(M.icosphere((0, 0, 0), r, 4)) / (4 / 3 * math.pi * r ** 3) - 1) < 0.005
    cr, ln = 0.05, math.sqrt(0.3 ** 2 + 0.1 ** 2)
    vol = math.pi * cr * cr * ln + 4 / 3 * math.pi * cr ** 3
    assert abs(M.signed_volume(M.capsule((0, 0, 0), (0, 0.3, 0.1), cr)) / vol - 1) < 0.01
    ec = math.pi * 0.17 * 0.11 * (1.38 - 0.85) + 4 / 3 * math.pi * 0.17 * 0.11 * 0.08
    assert abs(M.signed_volume(M.elliptic_capsule(0.85, 1.38, 0.17, 0.11, 0.08)) / ec - 1) < 0.01
    assert abs(M.signed_volume(M.box((0, 0, 0), (0.5, 0.05, 0.25))) - 8 * 0.5 * 0.05 * 0.25) < 1e-12


def test_test_body_components():
    body = M.test_body()
    assert len(body) == 5 and all(M.is_closed_manifold(c) for c in body)
    assert all(M.is_closed_manifold(c) for c in M.capsule_union_body())


@pytest.fixture(scope="module")
def sphere_field(oracle_mod):
    return oracle_mod.bake([M.icosphere((0, 0, 0), 0.1, 4)])


def test_sphere_distance_accuracy(sphere_field):
    dirs, rng = _directions(7, 2000)
    r = 0.1 + rng.uniform(-0.015, 0.015, 2000)
    p = dirs * r[:, None]
    assert np.abs(sphere_field.sample(p) - (r - 0.1)).max() <= 0.001


def test_sign_inside_outside(sphere_field):
    assert abs(sphere_field.sample(np.zeros((1, 3)))[0] + 0.02) <= 1e-6
    assert abs(sphere_field.sample(np.array([[0.15, 0, 0]]))[0] - 0.02) <= 1e-6


def test_gradient_points_outward(sphere_field):
    dirs, _ = _directions(11, 200)
    for d in dirs:
        g = _gradient(sphere_field, 0.105 * d)
        assert abs(np.linalg.norm(g) - 1) <= 1e-9
        assert math.degrees(math.acos(np.clip(g @ d, -1, 1))) <= 5.0


def test_union_is_min(oracle_mod):
    f = oracle_mod.bake([M.icosphere((0.08, 0, 0), 0.1, 4), M.icosphere((-0.08, 0, 0), 0.1, 4)])
    assert f.sample(np.zeros((1, 3)))[0] < 0
    assert abs(f.sample(np.array([[0.08, 0, 0.115]]))[0] - 0.015) <= 0.001
    crease = np.array([0.0, 0.0, 0.085])
    expected = np.linalg.norm(crease - np.array([0.08, 0, 0])) - 0.1
    v = f.sample(crease[None])[0]
    assert v > 0 and v <= expected + 1e-6 and abs(v - expected) <= 0.002


def test_outside_grid_is_far_outside(sphere_field):
    f = sphere_field
    assert f.sample(np.array([[10.0, 10, 10]]))[0] == f.band
    lo = f.origin
    hi = f.origin + f.cell_size * (np.asarray(f.dims) - 1)
    for a in range(3):
        below, above = 0.5 * (lo + hi), 0.5 * (lo + hi)
        below[a], above[a] = lo[a] - 1e-6, hi[a] + 1e-6
        assert f.sample(below[None])[0] == f.band and f.sample(above[None])[0] == f.band


def test_rejects_open_mesh(oracle_mod):
    m = M.icosphere((0, 0, 0), 0.1, 2)
    m.triangles = m.triangles[:-1]
    with pytest.raises(ValueError, match="not a closed manifold"):
        oracle_mod.bake([m])


def test_test_body_bake(oracle_mod):
    t0 = time.perf_counter()
    f = oracle_mod.bake(M.test_body())
    assert time.perf_counter() - t0 < 10.0  # the reference's bar is 2 s for its own build (test_collision_perf.cpp)
    assert f.sample(np.array([[0.0, 1.2, 0.0]]))[0] < 0  # inside the torso
