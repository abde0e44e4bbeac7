"""Batched drapes (include/drape_batch.h) through the C ABI, against one drape_solver per garment.

A batch garment runs the same kernels as a single solver built from its scene. What changes is the grouping of the
FP64 reductions (a garment's solve group has fewer blocks than a solver's grid) and, with the autotuner's product
schemes (slot-parallel, or 2, 4, 8 lanes per row), the order of each row's FP32 sums in the SpMV. FP64 regrouping
leaves the FP32-rounded PCG scalars as they are, so those runs track each other closely; an FP32 difference, like
any rounding difference, grows over frames on these drops (contact activation, Armijo halvings and PCG iteration
counts are discrete decisions): on the tubes here a 5e-7 m difference after one frame reaches centimetres after
three. Bars:
  - eight frames of three uneven garments on their own bodies (PCG converged to 1e-6, the single solver's product
    scheme): 1e-4 m from the single solvers, the same Newton iteration and substep counts;
  - graph replay and direct launches: bit-identical;
  - autotuning leaves the state as it was (bit-identical) and picks one of its variants;
  - every solve variant: one frame within 1e-5 m of the default (the one-frame trajectory bar of the parity tests),
    the same PCG iteration counts; block sizes alone regroup only FP64 sums;
  - the learned preconditioner with an identity network tracks block-Jacobi (1e-4 m after two frames);
  - drape to rest: the batch runner settles the garments the single solver settles, with the same assembly length
    (two frames) and a settle frame count within 25 %.
"""
import numpy as np
import pytest

from drape_b200 import batch as BT
from drape_b200 import learned
from drape_b200 import scenes as S
from drape_b200.scene import Scene, Settings

pytestmark = pytest.mark.gpu

ASSEMBLING, SETTLING = 0, 1


def _scenes(tolerance=1e-6, cap=1000):
    st = Settings(cg_tolerance=tolerance, max_cg_iterations=cap)
    return [S.tube_variant(11, 1500, field_n=48, settings=st),
            S.sheet_on_sphere(20, cg_tolerance=tolerance, max_cg=cap),
            S.tube_variant(12, 3200, field_n=64, settings=Settings(cg_tolerance=tolerance, max_cg_iterations=cap))]


def _batch(gpu, scenes, precond=None, like_single=False):
    """A built batch; like_single: the single solver's product scheme (2 lanes per row), so that both do the same FP32
    arithmetic and differ only in the grouping of FP64 sums."""
    b = BT.BatchSolver(0)
    for sc in scenes:
        b.add(sc)
    if precond is not None:
        b.set_precond(precond)
    b.build()
    if like_single:
        b.set_tuning(2, 1024)
    return b


def _frames(stepper, phase_fn, frames=8, settle_at=4):
    for f in range(frames):
        if f == 0:
            phase_fn(ASSEMBLING)
        if f == settle_at:
            phase_fn(SETTLING)
        stepper()


def test_batch_tracks_single_solvers(gpu):
    scenes = _scenes()
    b = _batch(gpu, scenes, like_single=True)
    _frames(lambda: b.step(1 / 60, 1, 2), lambda ph: [b.set_phase(i, ph) for i in range(len(scenes))])
    for i, sc in enumerate(scenes):
        s = gpu.CudaSolver(0)
        s.build(sc)
        gid = sc.garments[0].id
        _frames(lambda: s.step(1 / 60, 1, 2), lambda ph: s.set_phase(gid, ph))
        dev = np.abs(b.positions(i).astype(np.float64) - s.positions()).max()
        assert dev < 1e-4, (i, dev)
        assert b.counters(i).newton_iterations == s.counters().newton_iterations
        assert b.counters(i).substeps == s.counters().substeps


def test_batch_stats_match_single_solver(gpu):
    scenes = _scenes()
    b = _batch(gpu, scenes, like_single=True)
    b.step(1 / 60, 1, 2)
    for i, sc in enumerate(scenes):
        s = gpu.CudaSolver(0)
        s.build(sc)
        s.step(1 / 60, 1, 2)
        a, c = b.stats(i), s.stats()
        assert abs(a.kinetic_energy - c.kinetic_energy) <= 1e-3 * max(c.kinetic_energy, 1e-12)
        assert abs(a.max_seam_gap - c.max_seam_gap) <= 1e-5
        assert abs(a.max_body_penetration - c.max_body_penetration) <= 1e-5


def test_graph_replay_is_bit_identical_to_direct_launches(gpu):
    b = _batch(gpu, _scenes())
    b.save()
    for _ in range(3):
        b.step(1 / 60, 1, 2)
    graphed = [b.positions(i) for i in range(3)]
    assert b.profile_read()["graph_launches"] >= 3
    b.restore()
    b.profile(True)  # profiled frames launch directly
    for _ in range(3):
        b.step(1 / 60, 1, 2)
    p = b.profile_read()
    assert p["graph_launches"] == 0 and p["solve_launches"] == 6 and p["solve_ms"] > 0
    for i in range(3):
        assert np.array_equal(graphed[i], b.positions(i))


def test_autotune_keeps_the_state_and_picks_a_variant(gpu):
    b = _batch(gpu, _scenes())
    b.step(1 / 60, 1, 2)
    before = [b.positions(i) for i in range(3)]
    t = b.autotune(1)
    assert t["row_lanes"] in (0, 2, 4, 8) and t["block_threads"] in (256, 512, 1024) and t["variants_timed"] == 12
    assert t["ms_per_newton"] > 0
    for i in range(3):
        assert np.array_equal(before[i], b.positions(i))
    assert b.counters(0).newton_iterations == 0


@pytest.mark.parametrize("lanes,threads", [(0, 256), (2, 256), (4, 256), (8, 512), (0, 1024), (4, 1024)])
def test_every_variant_gives_the_same_frame(gpu, lanes, threads):
    ref = _batch(gpu, _scenes(1e-2, 50))
    b = _batch(gpu, _scenes(1e-2, 50))
    t = b.set_tuning(lanes, threads)
    assert (t["row_lanes"], t["block_threads"]) == (lanes, threads) and t["blocks"] > 0
    ref.step(1 / 60, 1, 2)
    b.step(1 / 60, 1, 2)
    for i in range(3):
        assert np.abs(ref.positions(i).astype(np.float64) - b.positions(i)).max() < 1e-5
        assert ref.counters(i).cg_iterations == b.counters(i).cg_iterations


def test_identity_network_tracks_jacobi_in_the_batch(gpu):
    a = _batch(gpu, _scenes())
    b = _batch(gpu, _scenes(), learned.LearnedPreconditioner(0))
    for x in (a, b):
        for i in range(3):
            x.set_phase(i, ASSEMBLING)
        x.step(1 / 60, 1, 2)
        x.step(1 / 60, 1, 2)
    for i in range(3):
        c = b.counters(i)
        assert c.learned_solves == c.newton_iterations > 0 and c.precond_fallbacks == 0
        assert np.abs(a.positions(i).astype(np.float64) - b.positions(i)).max() < 1e-4


def test_errors_map_to_reference_exceptions(gpu):
    b = BT.BatchSolver(0)
    with pytest.raises(gpu.CudaError, match="not built"):
        b.step(1 / 60, 1, 2)
    with pytest.raises(ValueError, match="exactly one garment"):
        b.add(Scene([S.sewn_pair(), S.centred_sheet(0.1, 0.02, 0.0)]))
    b.add(_scenes()[1])
    b.build()
    with pytest.raises(IndexError):
        b.positions(5)
    with pytest.raises(IndexError):
        b.set_phase(3, SETTLING)


def test_drape_to_rest_matches_single_solver_runs(gpu):
    scenes = [S.tube_10k(), S.seamed_tube(24, 30, field_n=64, field_cell=0.008, gid="small")]
    b = _batch(gpu, scenes, like_single=True)
    res, secs = b.drape_to_rest()
    assert len(res) == 2 and np.all(secs > 0)
    single = []
    for sc in scenes:
        s = gpu.CudaSolver(0)
        s.build(sc)
        single.append(s.drape_to_rest([sc.garments[0].id]))
    assert single[0].settled == 1  # the 10k tube settles
    for i, r in enumerate(single):
        assert res[i].settled == r.settled, (i, res[i].frames_run, r.frames_run)
        assert abs(res[i].assembly_seconds - r.assembly_seconds) <= 2 / 60 + 1e-9
        if r.settled:
            assert abs(res[i].frames_run - r.frames_run) <= 0.25 * r.frames_run, (res[i].frames_run, r.frames_run)
        st = b.stats(i)
        assert not st.has_non_finite and st.max_body_penetration <= 0.002
