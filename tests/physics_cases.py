"""The reference's analytic known-answer physics tests, restated on grid meshes, written once against the Solver
interface so they run on the oracle (CPU) and on the CUDA solver (GPU).

Sources: libs/sim/tests/test_cpu_solver.cpp (free fall, assembling, pins, strip strain, updateFabric, snapshot,
thin piece, ranges), test_body_collision.cpp (rest on sphere, pressed patch, tunnelling, starts inside, slope
friction), test_seams.cpp (gap after build, closing speed, hold when settling), test_bending.cpp (flat sheet stays
flat)."""
import math

import numpy as np
import pytest

from drape_b200 import scenes as S
from drape_b200.scene import Scene, Settings, jersey_fabric, stiff_fabric


def with_damping(f, d):
    f.damping = d
    return f


def run_until_still(s, dt, sub, its, rms, hold, max_seconds):
    """Steps until rmsSpeed < rms for hold consecutive frames; returns frames run or -1 (sim_test_utils.hpp:34-44)."""
    still = 0
    for f in range(1, int(math.ceil(max_seconds / dt)) + 1):
        s.step(dt, sub, its)
        still = still + 1 if s.stats().rms_speed < rms else 0
        if still >= hold:
            return f
    return -1


def free_fall(make):
    sc = Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, with_damping(jersey_fabric(), 0.0))])
    s = make()
    s.build(sc)
    before = np.asarray(s.positions(), np.float64)
    for _ in range(30):
        s.step(1 / 60, 10, 2)
    after = np.asarray(s.positions(), np.float64)
    assert np.allclose((after[:, 1] - before[:, 1]) / -1.22625, 1.0, atol=0.005)
    assert np.abs(after[:, 0] - before[:, 0]).max() <= 1e-5
    assert np.abs(after[:, 2] - before[:, 2]).max() <= 1e-5


def assembling_disables_gravity(make):
    sc = Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())])
    s = make()
    s.build(sc)
    s.set_phase("sheet", 0)
    before = np.asarray(s.positions(), np.float64)
    for _ in range(30):
        s.step(1 / 60, 10, 2)
    assert np.linalg.norm(np.asarray(s.positions(), np.float64) - before, axis=1).max() < 1e-6


def pins_hold(make):
    sc = Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())])
    sc.pins.append((0, tuple(sc.garments[0].initial_positions[0])))
    s = make()
    s.build(sc)
    for _ in range(60):
        s.step(1 / 60, 10, 2)
    assert np.linalg.norm(np.asarray(s.positions()[0], np.float64) - np.asarray(sc.pins[0][1])) < 1e-7


def strip_strain(make, grain, expected):
    sc = S.strip_scene(grain)
    s = make()
    s.build(sc)
    assert run_until_still(s, 1 / 60, 1, 2, 1e-5, 60, 30.0) > 0
    strain = S.measured_strain(np.asarray(s.positions(), np.float64), sc.garments[0].rest)
    assert strain == pytest.approx(expected, abs=0.05 * expected)


def update_fabric_changes_stiffness(make):
    f = with_damping(jersey_fabric(), 1.0)
    sc = S.strip_scene((1.0, 0.0), f)
    s = make()
    s.build(sc)
    assert run_until_still(s, 1 / 60, 1, 2, 1e-5, 60, 30.0) > 0
    f.stretch_warp = 800
    s.update_fabric("strip", [f])
    assert run_until_still(s, 1 / 60, 1, 2, 1e-5, 60, 30.0) > 0
    strain = S.measured_strain(np.asarray(s.positions(), np.float64), sc.garments[0].rest)
    assert strain == pytest.approx(0.0125, abs=0.05 * 0.0125)


def snapshot_restore_is_deterministic(make):
    sc = Scene([S.flat_garment("sheet", 0.2, 0.2, 0.02, jersey_fabric())])
    sc.pins.append((0, tuple(sc.garments[0].initial_positions[0])))
    s = make()
    s.build(sc)
    for _ in range(10):
        s.step(1 / 60, 10, 2)
    snap = s.snapshot()
    for _ in range(20):
        s.step(1 / 60, 10, 2)
    first = np.array(s.positions())
    s.restore(snap)
    for _ in range(20):
        s.step(1 / 60, 10, 2)
    assert np.array_equal(first, np.array(s.positions()))


def thin_piece_steps(make):
    sc = Scene([S.flat_garment("thin", 0.5, 0.02, 0.02, jersey_fabric())])
    s = make()
    s.build(sc)
    for _ in range(60):
        s.step(1 / 60, 10, 2)
    assert not s.stats().has_non_finite


def ranges_and_counts(make):
    sc = Scene([S.flat_garment("a", 0.1, 0.1, 0.02, jersey_fabric()),
                S.flat_garment("b", 0.2, 0.1, 0.02, jersey_fabric(), (0.5, 0.0, 0.0))])
    s = make()
    s.build(sc)
    ra, rb = s.range("a"), s.range("b")
    assert ra == (0, sc.garments[0].vertex_count)
    assert rb == (ra[1], sc.garments[1].vertex_count)
    assert s.particle_count() == ra[1] + rb[1]
    with pytest.raises(IndexError):
        s.range("zzz")


def rest_on_sphere(make):
    field = S.sphere_field()
    sc = Scene([S.centred_sheet(0.004, 0.004, 0.15 + 0.05)], field)
    s = make()
    s.build(sc)
    for _ in range(120):
        s.step(1 / 60, 1, 2)
    phi = field.sample(np.asarray(s.positions(), np.float64))
    assert np.abs(phi - S.K_CONTACT).max() <= 0.0005


def pressed_patch_stays_on_surface(make):
    field = S.sphere_field()
    g = S.centred_sheet(0.004, 0.004, 0.15 + S.K_CONTACT)
    sc = Scene([g], field, forces=[(i, (0.0, -1e-4, 0.0)) for i in range(g.vertex_count)])
    s = make()
    s.build(sc)
    for _ in range(30):
        s.step(1 / 60, 1, 2)
    assert s.stats().max_body_penetration <= 0.002
    assert np.abs(field.sample(np.asarray(s.positions(), np.float64)) - S.K_CONTACT).max() <= 0.0005


def fast_patch_cannot_tunnel(make):
    field = S.sphere_field()
    g = S.centred_sheet(0.004, 0.004, 0.15 + 0.015)
    sc = Scene([g], field, forces=[(i, (0.0, -3e-4, 0.0)) for i in range(g.vertex_count)])
    s = make()
    s.build(sc)
    for _ in range(10):
        s.step(1 / 60, 1, 2)
    assert s.stats().max_body_penetration <= 0.002
    assert np.abs(field.sample(np.asarray(s.positions(), np.float64)) - S.K_CONTACT).max() <= 0.0005


def starts_inside_is_resolved(make):
    sc = Scene([S.centred_sheet(0.6, 0.01, 0.15 - 0.01)], S.sphere_field())
    s = make()
    s.build(sc)
    assert s.stats().max_body_penetration > 0.005
    for _ in range(60):
        s.step(1 / 60, 1, 2)
    st = s.stats()
    assert not st.has_non_finite
    assert st.max_body_penetration <= 0.002


def slide_on_slope(make, friction):
    sc, uphill = S.slope_scene(friction)
    s = make()
    s.build(sc)
    c0 = np.asarray(s.positions(), np.float64).mean(axis=0)
    for _ in range(120):
        s.step(1 / 60, 1, 2)
    return float((np.asarray(s.positions(), np.float64).mean(axis=0) - c0) @ uphill)


def friction_holds_and_slides(make):
    assert abs(slide_on_slope(make, 0.5)) < 0.002
    assert slide_on_slope(make, 0.2) < -0.05


def seams_close(make):
    sc = Scene([S.sewn_pair()], settings=Settings(gravity=(0.0, 0.0, 0.0)))
    s = make()
    s.build(sc)
    assert s.stats().max_seam_gap == pytest.approx(0.1, abs=1e-6)
    s.set_phase("pair", 0)
    for _ in range(12):
        s.step(1 / 60, 10, 2)
    assert 0.047 <= s.stats().max_seam_gap <= 0.053
    for _ in range(18):
        s.step(1 / 60, 10, 2)
    assert s.stats().max_seam_gap < 0.001


def seams_hold_when_settling(make):
    g = S.sewn_pair()
    sc = Scene([g])
    V = g.vertex_count // 2
    for v in range(V):
        if g.rest[v, 0] <= 1e-9:
            sc.pins.append((v, tuple(g.initial_positions[v])))
    s = make()
    s.build(sc)
    s.set_phase("pair", 0)
    for _ in range(30):
        s.step(1 / 60, 10, 2)
    assert s.stats().max_seam_gap < 0.001
    s.set_phase("pair", 1)
    for _ in range(120):
        s.step(1 / 60, 2, 10)
    st = s.stats()
    assert st.max_seam_gap < 0.001
    assert not st.has_non_finite


def flat_sheet_stays_flat(make):
    sc = Scene([S.flat_garment("sheet", 0.2, 0.2, 0.01, stiff_fabric())], settings=Settings(gravity=(0.0, 0.0, 0.0)))
    s = make()
    s.build(sc)
    for _ in range(60):
        s.step(1 / 60, 2, 10)
    assert np.abs(np.asarray(s.positions(), np.float64)[:, 1]).max() < 1e-6


CASES = {
    "free_fall": free_fall,
    "assembling_disables_gravity": assembling_disables_gravity,
    "pins_hold": pins_hold,
    "strip_warp": lambda make: strip_strain(make, (1.0, 0.0), 0.025),
    "strip_weft": lambda make: strip_strain(make, (0.0, 1.0), 0.05),
    "update_fabric": update_fabric_changes_stiffness,
    "snapshot_restore": snapshot_restore_is_deterministic,
    "thin_piece": thin_piece_steps,
    "ranges": ranges_and_counts,
    "rest_on_sphere": rest_on_sphere,
    "pressed_patch": pressed_patch_stays_on_surface,
    "no_tunnelling": fast_patch_cannot_tunnel,
    "starts_inside": starts_inside_is_resolved,
    "slope_friction": friction_holds_and_slides,
    "seams_close": seams_close,
    "seams_hold": seams_hold_when_settling,
    "flat_stays_flat": flat_sheet_stays_flat,
}
