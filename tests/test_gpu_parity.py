"""Parity of the CUDA path (called through the C ABI) with the reference and the oracle.

Bars:
  - integer artefacts (slot maps, CSR pattern, term lists) and contact candidates: bit-exact;
  - one-frame trajectories against the reference's own 32-bit GPU algorithm (golden outputs of oracle/_ref):
    1e-5 m, the reference's Metal-vs-emulator bar (docs/superpowers/notes/2026-10-27-phase-b-handoff.md:53);
  - assembled Newton system against the FP64 oracle: 1e-4 relative (FP32 assembly);
  - PCG: the reference rig's convergence bar (test_kernels.cpp:212-234) and agreement with the oracle's FP64 solve.
"""
import os

import numpy as np
import pytest

from drape_b200 import scenes as S
from drape_b200.scene import Scene, Settings, jersey_fabric

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_kernels.npz")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def G():
    return np.load(GOLDEN)


def test_structure_bit_exact_through_device_solver(gpu, oracle_mod):
    for scene in (S.sheet_on_sphere(), S.tube_10k(), Scene([S.sewn_pair()])):
        s = gpu.CudaSolver(0)
        s.build(scene)
        o = oracle_mod.OracleSolver()
        o.build(scene)
        p, r = s.structure(), o.structure()
        for k in p:
            assert np.array_equal(p[k], r[k]), k


@pytest.mark.parametrize("case", ["sheet", "tube"])
def test_contact_candidates_bit_exact(gpu, G, case):
    """The contact-candidate flags, normals and plane offsets equal the reference's 32-bit k_contact_setup bit for bit
    on identical substep-start positions."""
    if case == "sheet":
        scene = S.sheet_on_sphere()
    else:
        scene = S.seamed_tube(16, 20, field_n=64, field_cell=0.008)
    s = gpu.CudaSolver(0)
    s.build(scene)
    x = G[f"contact_{case}_x"]
    near, nrm, off = s.contact_candidates(x)
    assert near.sum() > 0
    assert np.array_equal(near, G[f"contact_{case}_near"])
    sel = near == 1
    assert np.array_equal(nrm[sel], G[f"contact_{case}_normal"][sel])
    assert np.array_equal(off[sel], G[f"contact_{case}_offset"][sel])


def test_contact_candidates_match_oracle_away_from_threshold(gpu, oracle_mod, G):
    """Against the FP64 oracle the flags agree except where phi lies within float rounding of r + reach."""
    scene = S.seamed_tube(16, 20, field_n=64, field_cell=0.008)
    s = gpu.CudaSolver(0)
    s.build(scene)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    x = G["contact_tube_x"]
    near, _, _ = s.contact_candidates(x)
    onear, _, _ = o.contact_candidates(x.astype(np.float64))
    phi = scene.body.sample(x.astype(np.float64))
    thr = 0.003 + 0.5 * 0.0006 + 0.01
    clear = np.abs(phi - thr) > 1e-6
    assert np.array_equal(near[clear], onear[clear])


def _traj_scene(name):
    f = jersey_fabric()
    f.damping = 0
    return {
        "freefall": (Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, f)]), None),
        "strip": (S.strip_scene(), None),
        "patch": (Scene([S.centred_sheet(0.004, 0.004, 0.2)], S.sphere_field()), None),
        "sheet": (S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50), None),
        "pair": (Scene([S.sewn_pair()], settings=Settings(gravity=(0.0, 0.0, 0.0))), ("pair", 0)),
    }[name]


@pytest.mark.parametrize("name", ["freefall", "strip", "patch", "sheet", "pair"])
def test_trajectory_matches_reference_gpu_algorithm(gpu, G, name):
    scene, phase = _traj_scene(name)
    s = gpu.CudaSolver(0)
    s.build(scene)
    if phase:
        s.set_phase(*phase)
    for _ in range(int(G[f"traj_{name}_frames"])):
        s.step(1 / 60, int(G[f"traj_{name}_substeps"]), 2)
    dev = np.abs(s.positions().astype(np.float64) - G[f"traj_{name}"].astype(np.float64)).max()
    assert dev < 1e-5, dev


def test_assembled_system_matches_oracle(gpu, oracle_mod):
    """The first Newton system (gradient, block Hessian, active contacts) of a substep on the sheet resting on the
    sphere, against the FP64 oracle on identical float state."""
    scene = S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50)
    scene.garments[0].initial_positions[:, 1] -= 0.147  # start touching the sphere's top
    s = gpu.CudaSolver(0)
    s.build(scene)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    for _ in range(3):
        s.step(1 / 60, 1, 2)
    o.restore(s.snapshot())
    g = s.capture_system(1 / 60)
    r = o.capture_system(1 / 60)
    assert np.array_equal(g["active"], r["active"])
    assert g["active"].sum() > 0
    Bg, Br = g["blocks"].astype(np.float64), r["blocks"]
    assert np.linalg.norm(Bg - Br) <= 1e-4 * np.linalg.norm(Br)
    rows = np.repeat(np.arange(len(g["diag_slot"])), np.diff(g["row_start"].astype(np.int64)))
    per_row = np.sqrt(np.bincount(rows, weights=((Bg - Br) ** 2).sum(axis=(1, 2))))
    row_norm = np.sqrt(np.bincount(rows, weights=(Br ** 2).sum(axis=(1, 2))))
    assert np.all(per_row <= 1e-4 * row_norm + 1e-6)
    gg, gr = g["grad"].astype(np.float64), r["grad"]
    assert np.linalg.norm(gg - gr) <= 1e-3 * np.linalg.norm(gr) + 1e-9


def test_pcg_on_reference_rig(gpu, G):
    n = len(G["rig_row_start"]) - 1
    b = G["rig_b"]
    step, resid, its = gpu.pcg(G["rig_row_start"], G["rig_col_index"], G["rig_blocks"], G["rig_pinned"],
                               np.zeros(n, np.uint8), np.zeros((n, 3), np.float32), (-b).astype(np.float32), 50, 1e-2)
    A = G["rig_dense"]
    assert 0 < its <= 50
    assert its == int(G["rig_ref_iterations"])
    assert np.linalg.norm(A @ step.astype(np.float64).reshape(-1) - b.reshape(-1)) <= 1e-2 * np.linalg.norm(b) * 1.0001
    assert np.abs(step - G["rig_ref_step"]).max() <= 1e-5 * np.abs(G["rig_ref_step"]).max()
    assert np.all(step[G["rig_pinned"] == 1] == 0)


def test_pcg_contact_filter_removes_normal(gpu, G):
    """test_kernels.cpp:236-250: an active particle's step has no component along its contact normal."""
    n = len(G["rig_row_start"]) - 1
    nrm = np.zeros((n, 3), np.float32)
    nv = np.array([0.3, 0.9, -0.2])
    nrm[0] = nv / np.linalg.norm(nv)
    active = np.zeros(n, np.uint8)
    active[0] = 1
    grad = np.tile(np.array([0.5, -1.0, 0.25], np.float32), (n, 1))
    step, _, _ = gpu.pcg(G["rig_row_start"], G["rig_col_index"], G["rig_blocks"], G["rig_pinned"], active, nrm, grad,
                         1, 1e-2)
    assert abs(float(step[0].astype(np.float64) @ nrm[0])) <= 1e-7
    assert np.linalg.norm(step[0]) > 1e-3


def test_pcg_matches_oracle_on_sheet_system(gpu, oracle_mod):
    """The device PCG (FP32 vectors, FP64 dots) and the oracle's FP64 PCG on the same sheet-on-sphere system."""
    scene = S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50)
    scene.garments[0].initial_positions[:, 1] -= 0.147
    o = oracle_mod.OracleSolver()
    o.build(scene)
    for _ in range(3):
        o.step(1 / 60, 1, 2)
    sysm = o.capture_system(1 / 60)
    n = len(sysm["diag_slot"])
    pinned = np.zeros(n, np.uint8)
    for tol in (1e-2, 1e-5):
        so, ro, ito = oracle_mod.pcg(sysm["row_start"], sysm["col_index"], sysm["blocks"], pinned, sysm["active"],
                                     sysm["normals"], sysm["grad"], 200, tol)
        sg, rg, itg = gpu.pcg(sysm["row_start"], sysm["col_index"], sysm["blocks"].astype(np.float32), pinned,
                              sysm["active"], sysm["normals"].astype(np.float32), sysm["grad"].astype(np.float32), 200,
                              tol)
        # Both stop at a relative residual of tol. With FP32 vectors the attainable solution accuracy is about
        # cond(A) * 6e-8 (~1e-3 here), so below tol = 1e-2 the two solutions agree to that floor, not to tol.
        assert abs(itg - ito) <= max(2, ito // 10)
        assert np.linalg.norm(sg - so) <= max(5 * tol, 1e-2) * np.linalg.norm(so)


def test_bounded_barrier_returns_error_status(gpu):
    """A grid barrier that nobody releases gives up after its limit and reports status 1; the device stays usable."""
    assert gpu.test_barrier_timeout(0, 2, 20_000_000) == 1
    s = gpu.CudaSolver(0)
    s.build(Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())]))
    s.step(1 / 60, 1, 2)
    assert not s.stats().has_non_finite


def test_two_runs_bit_identical(gpu):
    scene = Scene([S.centred_sheet(0.2, 0.02, 0.17)], S.sphere_field())
    runs = []
    for _ in range(2):
        s = gpu.CudaSolver(0)
        s.build(scene)
        for _ in range(60):
            s.step(1 / 60, 1, 2)
        runs.append(s.positions())
    assert np.array_equal(runs[0], runs[1])


def test_snapshot_replay_bit_identical_in_contact(gpu):
    scene = Scene([S.centred_sheet(0.2, 0.02, 0.17)], S.sphere_field())
    s = gpu.CudaSolver(0)
    s.build(scene)
    for _ in range(60):
        s.step(1 / 60, 1, 2)
    snap = s.snapshot()
    for _ in range(20):
        s.step(1 / 60, 1, 2)
    first = s.positions()
    s.restore(snap)
    for _ in range(20):
        s.step(1 / 60, 1, 2)
    assert np.array_equal(first, s.positions())


def test_stats_match_oracle_on_same_state(gpu, oracle_mod):
    scene = S.seamed_tube(16, 20, field_n=64, field_cell=0.008)
    s = gpu.CudaSolver(0)
    s.build(scene)
    s.set_phase("tube", 0)
    for _ in range(10):
        s.step(1 / 60, 1, 2)
    o = oracle_mod.OracleSolver()
    o.build(scene)
    o.restore(s.snapshot())
    a, b = s.stats(), o.stats()
    assert a.has_non_finite == b.has_non_finite
    for k in ("kinetic_energy", "rms_speed", "max_seam_gap", "max_body_penetration"):
        assert getattr(a, k) == pytest.approx(getattr(b, k), rel=1e-6, abs=1e-12), k


def test_injected_failure_raises_and_recovers(gpu):
    s = gpu.CudaSolver(0)
    s.build(Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())]))
    s.inject_failure(1)
    s.step(1 / 60, 1, 2)
    with pytest.raises(gpu.CudaError, match="cuda"):
        s.step(1 / 60, 1, 2)
    s.inject_failure(-1)
    s.step(1 / 60, 1, 2)
    assert not s.stats().has_non_finite


def test_errors_map_to_reference_exceptions(gpu):
    s = gpu.CudaSolver(0)
    with pytest.raises(gpu.CudaError):
        s.step(1 / 60, 1, 2)  # not built
    s.build(Scene([S.flat_garment("sheet", 0.1, 0.1, 0.02, jersey_fabric())]))
    with pytest.raises(ValueError):
        s.read_positions(np.zeros((3, 3), np.float32))
    with pytest.raises(IndexError):
        s.set_phase("nope", 0)
    with pytest.raises(ValueError):
        s.update_fabric("sheet", [jersey_fabric(), jersey_fabric()])
    snap = s.snapshot()
    snap["positions"] = snap["positions"][:-1]
    snap["velocities"] = snap["velocities"][:-1]
    with pytest.raises(ValueError):
        s.restore(snap)
    from drape_b200.session import DrapeOptions
    for bad in (dict(snapshot_every=0), dict(substeps=0), dict(frame_dt=0.0)):
        with pytest.raises(ValueError, match="must be positive"):
            s.drape_to_rest(["sheet"], DrapeOptions(**bad).to_c())


def test_drape_to_rest_settles_the_10k_tube(gpu):
    """The 10k seamed tube settles (the FP64 oracle settles it in 221 frames)."""
    scene = S.tube_10k()
    s = gpu.CudaSolver(0)
    s.build(scene)
    res = s.drape_to_rest(["tube"])
    assert res.settled == 1 and res.retries == 0 and 0 < res.frames_run < 1200
    st = s.stats()
    assert not st.has_non_finite
    assert st.max_body_penetration <= 0.002


def test_drape_to_rest_ends_a_marginal_drape_in_a_terminal_state(gpu):
    """A 24 x 30 tube that the FP64 oracle does not settle within the 20 s limit either: the runner stops in one of
    its terminal states (timed out, or failed after max_retries doubled-substep retries) with a sane state."""
    scene = S.seamed_tube(24, 30, field_n=64, field_cell=0.008)
    s = gpu.CudaSolver(0)
    s.build(scene)
    res = s.drape_to_rest(["tube"])
    assert res.frames_run > 0
    assert res.settled == 1 or res.simulated_seconds >= 19.9 or (res.failed == 1 and res.retries == 3)
    st = s.stats()
    assert not st.has_non_finite
    assert st.max_body_penetration <= 0.002

@pytest.mark.gpu
def test_profile_solve_only_times_k_solve_alone(gpu):
    """drape_cuda_profile(s, 2): events around k_solve only (two a Newton iteration), every other kernel untimed."""
    s = gpu.CudaSolver(0)
    s.build(S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50))
    s.profile(True, solve_only=True)
    for _ in range(3):
        s.step(1 / 60, 1, 2)
    s.stats()
    p = s.profile_read()
    s.profile(False)
    assert p["launches"]["k_solve"] == 6 and p["milliseconds"]["k_solve"] > 0
    assert all(v == 0 for k, v in p["launches"].items() if k != "k_solve")
    s.profile(True)
    s.step(1 / 60, 1, 2)
    p = s.profile_read()
    assert p["launches"]["k_solve"] == 2 and p["launches"]["k_begin"] == 1 and p["launches"]["k_assemble"] == 4


def _drape_with(gpu, scene, gid, frames_per_wait, direct=False):
    from drape_b200.session import DrapeOptions
    s = gpu.CudaSolver(0)
    s.build(scene)
    if direct:
        s.profile(True)  # timed launches, one by one, instead of the frame graphs
    res = s.drape_to_rest([gid], DrapeOptions(frames_per_wait=frames_per_wait).to_c())
    fields = {f: getattr(res, f) for f, _ in type(res)._fields_}
    return fields, s.snapshot()


@pytest.mark.parametrize("scene_name", ["tube_10k", "marginal"])
def test_drape_to_rest_frame_batches_match_one_frame_per_wait(gpu, scene_name):
    """frames_per_wait only changes how often the host waits: batches of 10 and of 7 frames (whose discarded frames
    are replayed where a decision falls inside a batch) end in the same state, bit for bit, with the same result as
    one frame per wait. The reference run launches every kernel directly (profiling on), the batched runs replay
    frame graphs, so the graphs are checked too. The 10k tube covers the phase change and the settle hold; the
    marginal tube the time limit or the restore-and-retry path."""
    scene = S.tube_10k() if scene_name == "tube_10k" else S.seamed_tube(24, 30, field_n=64, field_cell=0.008)
    ref_res, ref_snap = _drape_with(gpu, scene, "tube", 1, direct=True)
    assert ref_res["frames_run"] > 0
    for fpw in (10, 7):
        res, snap = _drape_with(gpu, scene, "tube", fpw)
        assert res == ref_res, (fpw, res, ref_res)
        for key in ("positions", "velocities", "contact_force", "phases", "assembly_time", "seam_start_gap"):
            assert np.array_equal(snap[key], ref_snap[key]), (fpw, key)


def test_host_wait_mode_does_not_change_results(gpu):
    """The host's wait for the stream (poll only, or poll then sleep) changes when the host sees the work done, never
    the work: 20 frames of the sheet drop give bit-identical positions either way."""
    out = []
    for spin in (2**32 - 1, 0, 200):
        s = gpu.CudaSolver(0)
        s.set_host_wait(spin)
        s.build(S.sheet_on_sphere(cg_tolerance=1e-2, max_cg=50))
        for _ in range(20):
            s.step(1 / 60, 1, 2)
        out.append(s.positions())
        s.close()
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
