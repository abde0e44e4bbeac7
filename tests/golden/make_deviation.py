"""Generates tests/golden/deviation.npz: the oracle's results on the workloads' configurations, against which the CUDA
path's deviation is reported (tests and bench.py's `deviation` object).

The oracle is the CPU restatement of the reference CpuSolver (oracle/), run in its two modes: faithful (float particle
state, double solve: the reference CpuSolver) and full FP64. For every configuration it records the end positions of
both modes and the oracle's own self-spread: the distance between the faithful run and a faithful run whose start
positions moved by a seeded uniform +-1 um per coordinate, the reference's yardstick for what a 1 mm bar means on a
scene (libs/sim/tests/test_gpu_parity.cpp:12-20, :55-63).

Configurations (the scenes of drape_b200.scenes):
  c1        the 40 x 40 sheet dropped on the sphere, 120 frames, PCG tolerance 1e-6 (cap 3000), FP64
  c2        the 10k seamed tube from its start, 300 frames: Assembling for the frames the oracle's own drape assembled,
            then Settling
  c3        the 60k seamed tube, 60 frames continued from the state the faithful oracle drapes it to rest in (stored
            as c3_start_*)
  c3drape   the 60k tube's whole drape to rest from its start (DrapeSession criterion): the settled shapes
Each frame is one substep with two Newton iterations, dt = 1/60 s.

Run: python tests/golden/make_deviation.py   (uses all host cores; the oracle's results do not depend on the count)
"""
from __future__ import annotations

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "drape-2_b200"))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from drape_b200 import scenes as S  # noqa: E402
from drape_b200 import session as SS  # noqa: E402

OUT = os.path.join(HERE, "deviation.npz")
SNAP_KEYS = ("positions", "velocities", "phases", "assembly_time", "seam_start_gap", "contact_force")
PERTURB = 1e-6


def perturbed(snap: dict, amount: float = PERTURB, seed: int = 1) -> dict:
    """The snapshot with every start coordinate moved by amount * uniform(-1, 1) (numpy default_rng(seed))."""
    s = dict(snap)
    x = np.asarray(s["positions"], np.float64)
    s["positions"] = (x + amount * np.random.default_rng(seed).uniform(-1.0, 1.0, x.shape)).astype(np.float32)
    return s


def run(scene, frames: int, fp64: bool = False, start: dict | None = None, perturb: bool = False,
        settle_after: int | None = None) -> np.ndarray:
    """End positions after `frames` frames; `settle_after`: the frame at which the garments switch from Assembling
    (set at frame 0) to Settling."""
    o = O.OracleSolver(full_fp64=fp64)
    o.build(scene)
    if start is not None:
        o.restore(start)
    if perturb:
        o.restore(perturbed(o.snapshot()))
    gids = [g.id for g in scene.garments]
    for f in range(frames):
        if settle_after is not None and f == 0:
            for g in gids:
                o.set_phase(g, 0)
        if settle_after is not None and f == settle_after:
            for g in gids:
                o.set_phase(g, 1)
        o.step(1.0 / 60.0, 1, 2)
    return o.positions()


def drape(scene, fp64: bool = False, perturb: bool = False):
    o = O.OracleSolver(full_fp64=fp64)
    o.build(scene)
    if perturb:
        o.restore(perturbed(o.snapshot()))
    res = SS.drape_to_rest(o, [g.id for g in scene.garments])
    return o, res


def distances(a: np.ndarray, b: np.ndarray):
    d = np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=1)
    return float(d.max()), float(np.sqrt(np.mean(d * d)))


def record(out: dict, name: str, faithful, fp64, spread) -> None:
    out[f"{name}_faithful"] = np.asarray(faithful, np.float32)
    out[f"{name}_fp64"] = np.asarray(fp64, np.float32)
    out[f"{name}_spread_max"], out[f"{name}_spread_rms"] = distances(spread, faithful)
    out[f"{name}_faithful_vs_fp64_max"], out[f"{name}_faithful_vs_fp64_rms"] = distances(faithful, fp64)
    print(name, "spread %.3f mm, faithful vs fp64 %.3f mm" % (1e3 * out[f"{name}_spread_max"],
                                                             1e3 * out[f"{name}_faithful_vs_fp64_max"]), flush=True)


def main() -> None:
    O.lib().oracle_set_threads(0)
    out: dict = {"perturbation_m": PERTURB}
    t0 = time.perf_counter()
    # c1: sheet on sphere, FP64, tolerance 1e-6.
    sc = S.sheet_on_sphere(cg_tolerance=1e-6, max_cg=3000)
    record(out, "c1", run(sc, 120), run(sc, 120, fp64=True), run(sc, 120, perturb=True))
    out["c1_frames"], out["c1_cg_tolerance"], out["c1_max_cg"] = 120, 1e-6, 3000
    # c2: 10k tube from its start with the oracle's own assembly length.
    sc = S.tube_10k()
    _, res = drape(sc)
    asm = int(round(res.assembly_seconds * 60.0))
    record(out, "c2", run(sc, 300, settle_after=asm), run(sc, 300, fp64=True, settle_after=asm),
           run(sc, 300, perturb=True, settle_after=asm))
    out["c2_frames"], out["c2_assembly_frames"] = 300, asm
    # c3: the 60k tube's drape to rest (faithful), continued 60 frames.
    sc = S.tube_60k()
    o, res = drape(sc)
    settled = o.snapshot()
    for k in SNAP_KEYS:
        out[f"c3_start_{k}"] = settled[k]
    out["c3_start_frames"] = int(res.frames_run)
    record(out, "c3", run(sc, 60, start=settled), run(sc, 60, fp64=True, start=settled),
           run(sc, 60, start=settled, perturb=True))
    out["c3_frames"] = 60
    # c3drape: the whole drape's settled shape (faithful = the c3 start), FP64 and from a perturbed start.
    o64, res64 = drape(sc, fp64=True)
    op, resp = drape(sc, perturb=True)
    record(out, "c3drape", settled["positions"], o64.positions(), op.positions())
    out["c3drape_frames_faithful"], out["c3drape_frames_fp64"] = int(res.frames_run), int(res64.frames_run)
    out["c3drape_frames_perturbed"] = int(resp.frames_run)
    out["c3drape_settled"] = bool(res.settled and res64.settled and resp.settled)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} in {time.perf_counter() - t0:.0f} s")


if __name__ == "__main__":
    main()
