#!/usr/bin/env python
"""Benchmark of the cloth solver's Newton-step hot path on B200: drape settle time.

One step = one drape of the seamed-tube workload to rest, run by the solver's drape runner (DrapeSession semantics,
libs/sim/src/drape_session.cpp:32-95: Assembling until the seams close, then Settling until the RMS speed stays below
2 mm/s for 60 frames). Step k drapes start state k mod 16: the workload's own (k = 0) or one with every coordinate
moved by a seeded uniform +-1 um. The metric is the mean device time to settle one drape; PCG iterations per Newton
step are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference] [--workload tube60k|tube10k]

--impl cuda (default): the CUDA library through its C ABI, inputs resident in HBM (value) and through the full
  host-buffer path (e2e: build from host arrays, drape, read positions back). For N > 1 every rank drapes its own
  replica (one drape does not shard); value is the slowest rank's mean settle time.
--impl reference: the reference solver's CPU algorithm (the oracle's restatement of CpuSolver, float particle state
  and double solve, its loops spread over all host threads with results identical to one thread) drapes the
  workload's own start state to rest once, timed whole: the K steps are K consecutive slices of that one drape's
  frames, so value is the measured wall time of the whole CPU drape.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "drape-2_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "drape settle s & PCG iters/step: learned vs Jacobi precond, same GPU, ≤1mm dev"
WORKLOADS = {
    "tube60k": dict(desc="seamed tube drape to rest: 2 panels 154x195 (60,060 particles, 118,728 triangles), seams "
                         "k=1e4 N/m along both side edges, capsule-union body sampled to a 256^3 FP32 field at 3 mm, "
                         "jersey fabric mu=0.4, dt=1/60 s, 1 substep, 2 Newton iterations, PCG cap 50 / tol 1e-2",
                    particles=60060),
    "tube10k": dict(desc="seamed tube drape to rest: 2 panels 63x80 (10,080 particles), 128^3 field at 6 mm, "
                         "jersey mu=0.4, dt=1/60 s, 1 substep, 2 Newton iterations, PCG cap 50 / tol 1e-2",
                    particles=10080),
}
SETTLE_FIXTURE = os.path.join(ROOT, "tests", "golden", "settle_frames.json")
# Drapes per timed step: the workload's own start state and fifteen copies with every coordinate moved by a seeded
# uniform +-1 um. The settle frame count of one start state is a first-passage time of an RMS speed that hovers at the
# 2 mm/s threshold for hundreds of frames (332-1110 frames over such start states on the 60k tube), so one drape
# alone does not measure the solver.
SEEDS = 16
SEED_DESC = ("step k drapes start state k mod 16: the workload's own (0) or one with every coordinate moved by uniform "
             "+-1 um (numpy default_rng(seed), seeds 1-15); value and e2e are means over all of them")


def seeded_positions(base32: np.ndarray, seed: int) -> np.ndarray:
    """Start positions of seed `seed`: the workload's own (0) or moved by a seeded uniform +-1 um (FP32)."""
    if seed == 0:
        return base32
    rng = np.random.default_rng(seed)
    return (base32 + rng.uniform(-1e-6, 1e-6, base32.shape).astype(np.float32)).astype(np.float32)


def make_scene(workload: str):
    from drape_b200 import scenes as S
    return S.tube_60k() if workload == "tube60k" else S.tube_10k()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def algorithmic_bytes(st: dict) -> dict:
    """Algorithmic bytes (FP32 vectors at 12 B per vec3, 36 B blocks, 4 B indices):
    SpMV = 40 B per block slot + 44 B per particle; one Jacobi PCG iteration = SpMV + 156 B per particle;
    one FP64 energy pass reads its inputs: 48 B per stretch term, 32 per hinge, 16 per seam, 96 per particle."""
    n, B = st["n"], st["B"]
    spmv = 40 * B + 44 * n
    pcg_iter = spmv + 156 * n
    energy = 48 * st["S"] + 32 * st["H"] + 16 * st["K"] + 96 * n
    return dict(spmv=spmv, pcg_iter=pcg_iter, energy=energy)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str, period_ms: int = 200):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", str(period_ms), "-i", gpu_id], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons, masks, power = [], [], set(), {}, []
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
            masks[parts[4]] = masks.get(parts[4], 0) + 1
            try:
                power.append(float(parts[3]))
            except ValueError:
                pass
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "sm_mhz_min": min(sm) if sm else None,
                "power_w_max": max(power) if power else None, "active_masks": masks}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_drape(workload: str, steps: int, warmup_frames: int, threads: int = 0) -> dict:
    """The reference CPU path (the oracle's faithful restatement of CpuSolver: float particle state, double solve,
    block-Jacobi PCG with the workload's cap and tolerance) drapes the workload's own start state to rest, timed whole
    on the host. Its loops run on `threads` host threads (0: all); the per-slot, per-particle and energy/dot sums keep
    the serial order, so the drape is the single-threaded one bit for bit. `warmup_frames` frames of a separate solver
    run first, untimed. Returns the wall time, the frame count, per-frame wall times folded into `steps` consecutive
    slices of equal frame count, the counters and the threads used."""
    import oracle as O
    from drape_b200 import session as SS
    L = O.lib()
    L.oracle_set_threads(threads)
    used = int(L.oracle_threads())
    scene = make_scene(workload)
    gid = scene.garments[0].id
    if warmup_frames > 0:
        w = O.OracleSolver()
        w.build(scene)
        w.set_phase(gid, 0)
        for _ in range(warmup_frames):
            w.step(1.0 / 60.0, 1, 2)
        del w
    o = O.OracleSolver()
    o.build(scene)
    sess = SS.DrapeSession(o, [gid])
    frame_s = []
    t0 = time.perf_counter()
    while not sess.finished():
        f0 = time.perf_counter()
        sess.advance()
        frame_s.append(time.perf_counter() - f0)
    total = time.perf_counter() - t0
    c = o.counters()
    k = max(1, steps)
    bounds = [round(i * len(frame_s) / k) for i in range(k + 1)]
    step_s = [float(sum(frame_s[bounds[i]:bounds[i + 1]])) for i in range(k)]
    r = sess.result
    return {"seconds": total, "frames": int(r.frames_run), "settled": bool(r.settled), "step_s": step_s,
            "newton_iterations": int(c.newton_iterations), "cg_iterations": int(c.cg_iterations),
            "line_search_halvings": int(c.line_search_halvings), "threads": used, "cpu": cpu_model(),
            "host_cpus": os.cpu_count()}


def run_reference(args):
    """The reference CPU path timed whole: one drape of the workload's own start state to rest (see reference_drape).
    Under torchrun only rank 0 runs it."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    r = reference_drape(args.workload, args.steps, args.warmup)
    value = r["seconds"]
    sample = (f"one whole drape of the workload's own start state to rest: {r['frames']} frames, settled "
              f"{r['settled']}, timed from its first frame to the frame that settles it, on {r['threads']} host "
              f"threads ({r['cpu']}, {r['host_cpus']} logical CPUs); the {args.steps} steps are consecutive slices "
              f"of its frames")
    line = {
        "metric": METRIC, "value": value, "unit": "s", "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1000.0 / max(1, args.steps), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"],
                   "solver": "CpuSolver restatement (float particle state, double solve), block-Jacobi PCG",
                   "step": "1/K of one whole CPU drape's frames (the K steps together are the drape, timed whole); "
                           "warm-up: W frames of a separate solver"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": r["threads"], "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "frames_to_settle": r["frames"], "settled": r["settled"],
        "step_s": [round(t, 3) for t in r["step_s"]],
        "pcg_iters_per_newton": {"mean": r["cg_iterations"] / max(1, r["newton_iterations"]), "cap": 50},
        "line_search_halvings": r["line_search_halvings"],
    }
    print(json.dumps(line))
    return 0


def network_forward(s, args, frames: int = 10) -> dict:
    """Device time of the learned preconditioner's network forward inside the 60k drape (the inference path:
    k_scale, k_features, k_slot_encode, k_node x 5, k_message x 4, k_output_rows), from `frames` more frames of the
    learned solver `s` with every kernel timed by CUDA events, beside its algorithmic bytes: per block slot 112 B of
    features (block 36, column 4, C_j 36, e 32, code 4), 608 B of slot encoding (e 32 read, E 512 and F 64 written),
    260 B per layer of messages (E 128, P_j 128, code 4) and 130 B of output (code and row 8, L 36 written, F 48 and
    Q_i, Q_j, C_i 108 on the lower live slots, about 55 %); per particle 72 B of scaling (diagonal block, C), 76 B of
    node features (C_i, row bounds, f), 136 B per layer of messages (row bounds, a) and 2336 B of node GEMMs (the
    encoder: f 32 read, h 128 and P 128 written; each layer's update: h 128 and a 128 read, h' 128 and P or Q 128
    written)."""
    st = s.structure()
    n, B = len(st["diag_slot"]), len(st["col_index"])
    s.profile(True)
    for _ in range(frames):
        s.step(1.0 / 60.0, 1, 2)
    p = s.profile_read()
    s.profile(False)
    launches = max(1, p["launches"]["net_forward"])
    ms = p["milliseconds"]["net_forward"] / launches
    algo = B * (112 + 608 + 4 * 260 + 130) + n * (72 + 76 + 4 * 136 + 288 + 4 * 512)
    peak, kind = measured_peaks()
    gbs = algo / (ms / 1e3) / 1e9 if ms > 0 else None
    # Tensor-core work (BF16 MMAs, FP32 accumulation): per slot the edge encoder (16 -> 64), the four layers' slot terms
    # and the output layer's (64 -> 256 + 16); per particle the node encoder and P^0 (16 -> 64 -> 64) and each layer's
    # update and next node term (128 -> 64 -> 64, the last 128 -> 64 -> 32).
    flops = 2 * B * (16 * 64 + 64 * 256 + 64 * 16) + 2 * n * (16 * 64 + 64 * 64 + 3 * (128 * 64 + 64 * 64)
                                                                + 128 * 64 + 64 * 32)
    tf = flops / (ms / 1e3) / 1e12 if ms > 0 else None
    bf16_peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16_peak = float(json.load(f)["bf16_tflops"])
    except (OSError, KeyError, ValueError):
        bf16_peak = 1590.0
    return {"ms_per_forward": ms, "forwards": launches, "particles": n, "block_slots": B,
            "algorithmic_bytes": algo, "achieved_gbs": gbs, "peak_gbs": peak, "peak_source": kind,
            "frac": gbs / peak if gbs else None,
            "tensor": {"flops": flops, "achieved_tflops": tf, "peak_bf16_tflops": bf16_peak,
                       "frac": tf / bf16_peak if tf else None,
                       "note": "the GEMMs are small (hidden 64); the forward is bound by memory, not the tensor pipe"},
            "note": f"{frames} frames of the learned 60k solver (every Newton iteration runs the network), CUDA events "
                    f"around each forward; the P_j gathers (4 x 128 B per slot) are served mostly from L2"}


def precond_leg(CU, device, args, flush, max_over_ranks, cap: int = 1000, tol: float = 1e-2, window: int = 120):
    """Block-Jacobi against the learned preconditioner on the same GPU and the same 60k tube, in two parts.
    settle: each drapes the workload's own start state to rest at the reference's PCG settings (cap 50, tolerance
      1e-2; L2 flushed first): settle seconds, frames, ms per frame, PCG iterations per Newton step;
    convergence: the first `window` frames from the same start with the PCG stopped by its tolerance (1e-2) under a
      cap of `cap` it is not meant to reach, so that PCG iterations per Newton step measure convergence, not the cap
      (the reference's cap of 50 binds on almost every 60k solve): iterations per Newton step (mean, p50, p95, max),
      whether the cap was reached, us per PCG iteration and ms per frame.
    The learned solver uses the shipped trained weights (drape_b200/weights/tube.npy) with the network run every
    `--refresh-every` Newton iterations; block-Jacobi stays its fallback."""
    import torch
    from drape_b200 import learned as LR
    from drape_b200 import scenes as S
    from drape_b200.scene import Settings

    def solver_for(name, scene):
        s = CU.CudaSolver(device)
        net = None
        if name == "learned":
            net = LR.LearnedPreconditioner(device, LR.load_weights("tube"))
            s.set_precond(net)
            s.set_precond_schedule(refresh_every=args.refresh_every)
        else:
            s.set_pcg_variant(args.pcg_variant)
        s.build(scene)
        return s, net

    def iters(s):
        h = np.asarray(s.cg_history(), np.int64)
        return {"mean": float(h.mean()) if len(h) else None, "p50": float(np.percentile(h, 50)) if len(h) else None,
                "p95": float(np.percentile(h, 95)) if len(h) else None, "max": int(h.max()) if len(h) else None}

    out = {"settle": {}, "convergence": {}}
    finals = {}
    for name in ("jacobi", "learned"):
        # settle, at the reference's settings
        s, net = solver_for(name, S.tube_60k())
        stream = torch.cuda.ExternalStream(s.stream_handle())
        s.reset_counters()
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = s.drape_to_rest(["tube"])
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        c = s.counters()
        finals[name] = s.positions().astype(np.float64)
        out["settle"][name] = {"settle_s": max_over_ranks(t), "frames": int(r.frames_run), "settled": bool(r.settled),
                               "ms_per_frame": 1000.0 * t / max(1, r.frames_run), "pcg_iters_per_newton": iters(s),
                               "us_per_pcg_iteration": c.pcg_nanoseconds / 1000.0 / max(1, c.cg_iterations)}
        s.close()
        if net is not None:
            net.close()
        # convergence, tolerance-driven
        s, net = solver_for(name, S.tube_60k(settings=Settings(max_cg_iterations=cap, cg_tolerance=tol)))
        stream = torch.cuda.ExternalStream(s.stream_handle())
        s.set_phase("tube", 0)
        s.reset_counters()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for f in range(window):
            if f == 20:
                s.set_phase("tube", 1)
            s.step(1.0 / 60.0, 1, 2)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        c = s.counters()
        it = iters(s)
        out["convergence"][name] = {"pcg_iters_per_newton": it, "cap_reached": bool(it["max"] is not None and it["max"] >= cap),
                                    "us_per_pcg_iteration": c.pcg_nanoseconds / 1000.0 / max(1, c.cg_iterations),
                                    "ms_per_frame": 1000.0 * t / window}
        if name == "learned":
            out["convergence"][name].update({"learned_solves": int(c.learned_solves),
                                             "jacobi_fallbacks": int(c.precond_fallbacks)})
            out["network_forward"] = network_forward(s, args)
        s.close()
        if net is not None:
            net.close()
    d = np.linalg.norm(finals["learned"] - finals["jacobi"], axis=1)
    js, ls = out["settle"]["jacobi"]["settle_s"], out["settle"]["learned"]["settle_s"]
    jm = out["convergence"]["jacobi"]["pcg_iters_per_newton"]["mean"]
    lm = out["convergence"]["learned"]["pcg_iters_per_newton"]["mean"]
    out.update({
        "workload": f"60k seamed tube; settle at the reference's PCG settings (cap 50, tol 1e-2) from the workload's "
                    f"own start state; convergence over its first {window} frames at tol {tol} with a cap of {cap}",
        "network_every_newton_iterations": args.refresh_every,
        "speedup_vs_jacobi": (js / ls) if ls else None,
        "pcg_iteration_ratio_at_tolerance": (jm / lm) if (jm and lm) else None,
        "settled_shape_learned_vs_jacobi_mm": {"max": 1e3 * float(d.max()), "rms": 1e3 * float(np.sqrt(np.mean(d * d)))},
    })
    return out


DEVIATION_FIXTURE = os.path.join(ROOT, "tests", "golden", "deviation.npz")


def _seam_gap_penetration(scene, x: np.ndarray):
    """Largest seam-pair distance and largest depth below the body's surface (m) of positions x, as SimModel::stats
    reports them (sim_model.cpp:222-241), from the scene's own seam pairs and sampled field."""
    x = np.asarray(x, np.float64)
    gap, off = 0.0, 0
    for g in scene.garments:
        if g.seam_pairs is not None and len(g.seam_pairs):
            sp = np.asarray(g.seam_pairs, np.int64)
            gap = max(gap, float(np.linalg.norm(x[off + sp[:, 0]] - x[off + sp[:, 1]], axis=1).max()))
        off += g.vertex_count
    pen = float(np.max(-scene.body.sample(x))) if scene.body is not None else 0.0
    return gap, pen


def deviation_leg(CU, device, jacobi_final=None, variant=0):
    """Deviation of the CUDA path from the oracle on the workloads' configurations, next to the oracle's own
    self-spread (its faithful run against a faithful run from a start moved by a seeded uniform +-1 um per coordinate:
    what a 1 mm bar can mean on that scene, libs/sim/tests/test_gpu_parity.cpp:12-20). The oracle's end states come
    from tests/golden/deviation.npz (made by tests/golden/make_deviation.py); the CUDA path runs the same frames here.
      c1       sheet on sphere, 120 frames, PCG tolerance 1e-6 (cap 3000)
      c2       10k tube from its start, 300 frames (Assembling for the oracle drape's assembly frames, then Settling)
      c3       60k tube, 60 frames continued from the faithful oracle's settled state (the reference's
               continue-from-settled parity case)
      c3drape  60k tube: the settled shape of the CUDA drape (the workload's own start state) against the oracle's
               settled shapes
    Each entry: max and RMS vertex distance to the faithful oracle (float state, double solve: the reference
    CpuSolver) and to the full-FP64 oracle, the seam gap and body penetration of each result, the self-spread."""
    from drape_b200 import scenes as S
    try:
        F = np.load(DEVIATION_FIXTURE)
    except OSError as e:
        return {"unavailable": f"no oracle fixture: {e}"}

    def dist(a, b):
        d = np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64), axis=1)
        return {"max_mm": 1e3 * float(d.max()), "rms_mm": 1e3 * float(np.sqrt(np.mean(d * d)))}

    def entry(name, scene, x, desc):
        fa, f64 = F[f"{name}_faithful"], F[f"{name}_fp64"]
        gap, pen = _seam_gap_penetration(scene, x)
        ogap, open_ = _seam_gap_penetration(scene, fa)
        gap64, pen64 = _seam_gap_penetration(scene, f64)
        return {"config": desc, "particles": int(len(x)),
                "vs_oracle_faithful": dist(x, fa), "vs_oracle_fp64": dist(x, f64),
                "oracle_self_spread": {"max_mm": 1e3 * float(F[f"{name}_spread_max"]),
                                       "rms_mm": 1e3 * float(F[f"{name}_spread_rms"])},
                "oracle_faithful_vs_fp64": {"max_mm": 1e3 * float(F[f"{name}_faithful_vs_fp64_max"]),
                                            "rms_mm": 1e3 * float(F[f"{name}_faithful_vs_fp64_rms"])},
                "seam_gap_mm": {"cuda": 1e3 * gap, "oracle_faithful": 1e3 * ogap, "oracle_fp64": 1e3 * gap64},
                "penetration_mm": {"cuda": 1e3 * pen, "oracle_faithful": 1e3 * open_, "oracle_fp64": 1e3 * pen64}}

    def run(scene, frames, start=None, settle_after=None):
        s = CU.CudaSolver(device)
        s.set_pcg_variant(variant)
        s.build(scene)
        if start is not None:
            s.restore(start)
        gids = [g.id for g in scene.garments]
        for f in range(frames):
            if settle_after is not None and f == 0:
                for g in gids:
                    s.set_phase(g, 0)  # Assembling
            if settle_after is not None and f == settle_after:
                for g in gids:
                    s.set_phase(g, 1)  # Settling
            s.step(1.0 / 60.0, 1, 2)
        x = s.positions().astype(np.float64)
        s.close()
        return x

    out = {}
    sc = S.sheet_on_sphere(cg_tolerance=1e-6, max_cg=3000)
    out["c1"] = entry("c1", sc, run(sc, 120), "sheet 40x40 dropped on the sphere, 120 frames, PCG tol 1e-6 cap 3000")
    sc = S.tube_10k()
    asm = int(F["c2_assembly_frames"])
    out["c2"] = entry("c2", sc, run(sc, 300, settle_after=asm),
                      f"10k seamed tube from its start, 300 frames (Assembling {asm} frames, then Settling)")
    sc = S.tube_60k()
    start = {k: F[f"c3_start_{k}"] for k in ("positions", "velocities", "phases", "assembly_time", "seam_start_gap",
                                              "contact_force")}
    out["c3"] = entry("c3", sc, run(sc, 60, start=start),
                      f"60k seamed tube, 60 frames continued from the faithful oracle's settled state "
                      f"({int(F['c3_start_frames'])} oracle frames to settle)")
    if jacobi_final is not None:
        out["c3drape"] = entry("c3drape", sc, jacobi_final,
                               "60k seamed tube: settled shape of the CUDA drape (block-Jacobi, the workload's own "
                               f"start) vs the oracle's settled shapes (faithful {int(F['c3drape_frames_faithful'])}, "
                               f"FP64 {int(F['c3drape_frames_fp64'])} frames)")
    out["bar_mm"] = 1.0
    out["pcg"] = {0: "reference order", 1: "pipelined", 2: "Chronopoulos-Gear"}[variant]
    return out


def spmv_leg(CU, solver, peak, tiles=12, reps=20):
    """The standalone block-CSR SpMV (drape_cuda_spmv_device) on an HBM-resident matrix: the 60k tube's first Newton
    system tiled block-diagonally `tiles` times (each tile's columns shifted), larger than the 126 MB L2, timed with
    CUDA events over `reps` launches on one stream. Algorithmic bytes: 40 per block slot + 44 per row."""
    import torch
    sysm = solver.capture_system(1.0 / 60.0)
    rs, ci = sysm["row_start"].astype(np.int64), sysm["col_index"].astype(np.int64)
    n1, b1 = len(rs) - 1, len(ci)
    n, B = n1 * tiles, b1 * tiles
    SP = (B + 31) // 32 * 32
    rs_all = np.concatenate([rs[:-1] + t * b1 for t in range(tiles)] + [np.array([B])]).astype(np.uint32)
    ci_all = np.concatenate([ci + t * n1 for t in range(tiles)]).astype(np.uint32)
    planes = np.zeros((9, SP), np.float32)
    planes[:, :B] = np.tile(sysm["blocks"].reshape(b1, 9).T, (1, tiles))
    dev = torch.device("cuda", torch.cuda.current_device())
    d_rs = torch.from_numpy(rs_all.view(np.int32)).to(dev)
    d_ci = torch.from_numpy(ci_all.view(np.int32)).to(dev)
    d_bl = torch.from_numpy(planes).to(dev)
    d_pin = torch.zeros(n, dtype=torch.uint8, device=dev)
    gen = torch.Generator(device="cpu").manual_seed(3)
    d_x = torch.randn((n, 4), generator=gen).to(dev)
    d_y = torch.zeros((n, 4), device=dev)
    L = CU.load()
    st = torch.cuda.current_stream()

    def launch():
        code = L.drape_cuda_spmv_device(n, d_rs.data_ptr(), d_ci.data_ptr(), d_bl.data_ptr(), SP, d_pin.data_ptr(),
                                        d_x.data_ptr(), d_y.data_ptr(), st.cuda_stream)
        if code != 0:
            raise RuntimeError(L.drape_cuda_last_error(None))

    for _ in range(3):
        launch()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        launch()
    b.record(st)
    b.synchronize()
    ms = a.elapsed_time(b) / reps
    # Check against a host product on a few rows of the first tile.
    y = d_y[:n1].cpu().numpy()
    bl = sysm["blocks"].reshape(b1, 3, 3).astype(np.float64)
    x = d_x[:n1, :3].cpu().numpy().astype(np.float64)
    err = 0.0
    for i in range(0, n1, max(1, n1 // 200)):
        ref = sum(bl[s] @ x[ci[s]] for s in range(rs[i], rs[i + 1]))
        err = max(err, float(np.abs(ref - y[i, :3]).max() / (np.abs(ref).max() + 1e-30)))
    algo = 40.0 * B + 44.0 * n
    achieved = algo / (ms / 1e3) / 1e9
    return {"kernel": "k_spmv", "rows": n, "block_slots": B, "matrix_mb": 36.0 * B / 1e6,
            "ms_per_launch": ms, "algorithmic_bytes_per_launch": algo, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "max_rel_error_vs_host": err,
            "workload": f"60k tube Newton system tiled {tiles}x block-diagonally (inputs larger than L2)"}


def batch_leg(args, device, world, rank, max_over_ranks, peak):
    """Batched drapes: the 64 uneven seeded tubes (2k-40k particles, each on its own seeded body), this rank's share
    (drape_b200.batch.shard), autotuned, draped to rest through the batch's graphed frames."""
    import torch
    from drape_b200 import batch as BT
    from drape_b200 import scenes as S
    scenes = S.batch_tubes(args.batch_garments)
    sizes = [sc.garments[0].vertex_count for sc in scenes]
    mine = BT.shard(sizes, world)[rank]
    b = BT.BatchSolver(device)
    for g in mine:
        b.add(scenes[g])
    b.build()
    G, N, B = b.size()
    b.save()
    tuning = b.autotune(2)
    stream = torch.cuda.ExternalStream(b.stream_handle())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.restore()
    b.reset_counters()
    b.profile(False)
    e0.record(stream)
    t0 = time.perf_counter()
    res, secs = b.drape_to_rest()
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) / 1000.0
    prof_graph = b.profile_read()
    total = max_over_ranks(max(wall, dev_s))
    # Roofline of the batch solve: 10 profiled frames from the initial state (direct launches, events per solve).
    b.restore()
    b.reset_counters()
    b.profile(True)
    for _ in range(10):
        b.step(1.0 / 60.0, 1, 2)
    p = b.profile_read()
    b.profile(False)
    achieved = p["pcg_bytes"] / (p["solve_ms"] / 1e3) / 1e9 if p["solve_ms"] > 0 else 0.0
    settled = [bool(r.settled) for r in res]
    frames = [int(r.frames_run) for r in res]
    settle_s = [float(t) for t, ok in zip(secs, settled) if ok]
    out = {
        "workload": f"{args.batch_garments} seamed tubes, particles log-uniform 2k-40k, each on its own seeded "
                    "capsule-union body (32^3-128^3 field), one persistent solve launch per Newton iteration, frames "
                    "replayed from a CUDA graph, autotuned solve variant, block-Jacobi PCG cap 50 / tol 1e-2",
        "garments": G, "particles": N, "block_slots": B, "rank_garments": len(mine),
        "settled_per_s": sum(settled) / total if total else None,
        "settled": int(sum(settled)), "unsettled": int(len(settled) - sum(settled)),
        "drape_s": total,
        "drapes_ended_per_s": args.batch_garments / total if total else None,
        "per_drape_settle_s": ({"median": float(np.median(settle_s)), "p90": float(np.percentile(settle_s, 90)),
                                "max": float(np.max(settle_s))} if settle_s else None),
        "frames": {"median_settled": float(np.median([f for f, ok in zip(frames, settled) if ok] or [0])),
                   "max": int(max(frames))},
        "unsettled_note": "garments still moving faster than 2 mm/s RMS at the 20 s limit (the tube geometry above ~15k "
                          "particles on these fields keeps a few mm/s of contact jitter); they end timed out, as the "
                          "reference's DrapeSession ends them; drapes_ended_per_s counts them, settled_per_s does not",
        "tuning": tuning, "graph_launches": int(prof_graph["graph_launches"]),
        "kernel_launches": int(prof_graph["kernel_launches"]),
        "roofline": {"kernel": "k_solve_batch", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None,
                     "avg_launch_ms": p["solve_ms"] / max(1, p["solve_launches"]),
                     "algorithmic_bytes_per_launch": p["pcg_bytes"] / max(1, p["solve_launches"]),
                     "sample": "10 frames from the initial state, profiled (direct launches)"},
    }
    b.close()
    return out


def bake_leg(peak):
    """The collision-field bake (drape_bake_field) of the reference's five-component test body at its default 4 mm
    cells (the reference's bar: under 2 s, test_collision_perf.cpp:11-19) and of the tube workloads' capsule-union
    body at 3 mm, device time per bake (mean of 3 after one warm-up), beside the oracle's serial restatement of the
    same bake on one host core."""
    import oracle as O
    from drape_b200 import bake as BK
    from drape_b200 import meshes as M
    out = {}
    for name, comps, opts in (("test_body_4mm", M.test_body(), BK.options()),
                              ("capsule_union_3mm", M.capsule_union_body(), BK.options(cell_size=0.003))):
        f = BK.bake_field(comps, opts)
        ms = []
        for _ in range(3):
            BK.bake_field(comps, opts)
            ms.append(BK.last_ms())
        t0 = time.perf_counter()
        ref = O.bake(comps, opts.cell_size, opts.padding, opts.band)
        cpu = time.perf_counter() - t0
        out[name] = {"triangles": M.triangle_count(comps), "samples": int(np.prod(f.dims)),
                     "device_ms": statistics.mean(ms), "cpu_oracle_ms_1_core": 1000.0 * cpu,
                     "bit_exact_vs_oracle": bool(np.array_equal(f.values, ref.values))}
    return out


def mesh_leg():
    """The pattern mesher (drape_mesh_build, host code; the reference's buildSimMesh): the tube workload's two
    0.55 x 0.7 m panels sewn along both side edges, meshed at the reference's three particle distances, wall time
    per mesh (best of 3) on one host core."""
    from drape_b200 import mesher as M
    a, b = M.rectangle_piece("front", 0.55, 0.7), M.rectangle_piece("back", 0.55, 0.7)
    pat = M.Pattern([a, b], [M.SeamSpec("left", M.segment_edge(a, "left", "left", False),
                                        M.segment_edge(b, "right", "right", True)),
                             M.SeamSpec("right", M.segment_edge(a, "right", "right", False),
                                        M.segment_edge(b, "left", "left", True))])
    out = {}
    for q in ("draft", "standard", "fine"):
        h = M.particle_distance(q)
        best, m = None, None
        for _ in range(3):
            t0 = time.perf_counter()
            m = M.build_sim_mesh(pat, h)
            dt = time.perf_counter() - t0
            best = dt if best is None else min(best, dt)
        out[q] = {"particle_distance_m": h, "vertices": int(len(m.rest)), "triangles": int(len(m.triangles)),
                  "seam_pairs": int(len(m.seam_pairs)), "ms": 1000.0 * best}
    return out


def run_profile_case(args):
    """One small case for an ncu capture (not a benchmark line): "spmv" times the standalone SpMV on the tiled tube
    system; "batch" builds the first --batch-garments tubes of the batched workload and runs --batch-frames frames
    (the first frame launches directly, the rest replay its CUDA graph); "bake" bakes the reference's test body;
    "drape" runs --batch-frames frames of the --workload drape (direct launches, from its own start state), and
    "drape_learned" the same with the learned preconditioner."""
    import torch
    from drape_b200 import cuda as CU
    torch.cuda.set_device(0)
    peak, _ = measured_peaks()
    if args.profile_case == "spmv":
        s = CU.CudaSolver(0)
        s.build(make_scene("tube60k"))
        print(json.dumps(spmv_leg(CU, s, peak, tiles=args.spmv_tiles)))
        return 0
    if args.profile_case == "learned":
        # One forward and one backward of the network (k_layer, k_bw_layer, ...) on a captured 10k-tube system.
        from drape_b200 import learned as LR
        s = CU.CudaSolver(0)
        s.build(make_scene("tube10k"))
        for _ in range(20):
            s.step(1.0 / 60.0, 1, 2)
        sysm = s.capture_system(1.0 / 60.0)
        n = len(sysm["diag_slot"])
        p = LR.LearnedPreconditioner(0, LR.load_weights("tube"))
        sid = p.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"], np.zeros(n, np.uint8),
                           sysm["active"], np.random.default_rng(0).standard_normal((1, n, 3)).astype(np.float32))
        p.forward(sid)
        loss, grad = p.loss_grad(sid)
        print(json.dumps({"case": "learned", "particles": n, "block_slots": int(len(sysm["col_index"])),
                          "loss": float(loss), "grad_norm": float(np.linalg.norm(grad))}))
        return 0
    if args.profile_case == "learned_inference":
        # The network's inference path (the solver's forward) on a captured --workload system, three times.
        from drape_b200 import learned as LR
        s = CU.CudaSolver(0)
        s.build(make_scene(args.workload))
        for _ in range(20):
            s.step(1.0 / 60.0, 1, 2)
        sysm = s.capture_system(1.0 / 60.0)
        n = len(sysm["diag_slot"])
        s.close()
        p = LR.LearnedPreconditioner(0, LR.load_weights("tube"))
        sid = p.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"], np.zeros(n, np.uint8),
                           sysm["active"], np.zeros((1, n, 3), np.float32))
        Ls = [p.forward_inference(sid) for _ in range(3)]
        print(json.dumps({"case": "learned_inference", "workload": args.workload, "particles": n,
                          "block_slots": int(len(sysm["col_index"])), "deterministic": bool(np.array_equal(Ls[0], Ls[2])),
                          "l_norm": float(np.linalg.norm(Ls[0]))}))
        return 0
    if args.profile_case in ("drape", "drape_learned"):
        s = CU.CudaSolver(0)
        s.set_pcg_variant(args.pcg_variant)
        if args.profile_case == "drape_learned":  # the shipped network every Newton iteration
            from drape_b200 import learned as LR
            net = LR.LearnedPreconditioner(0, LR.load_weights("tube"))
            s.set_precond(net)
        s.build(make_scene(args.workload))
        for _ in range(args.batch_frames):
            s.step(1.0 / 60.0, 1, 2)
        c = s.counters()
        print(json.dumps({"case": args.profile_case, "workload": args.workload, "frames": args.batch_frames,
                          "newton_iterations": int(c.newton_iterations), "cg_iterations": int(c.cg_iterations)}))
        return 0
    if args.profile_case == "bake":
        from drape_b200 import bake as BK
        from drape_b200 import meshes as M
        f = BK.bake_field(M.test_body())
        print(json.dumps({"case": "bake", "samples": int(np.prod(f.dims)), "device_ms": BK.last_ms()}))
        return 0
    from drape_b200 import batch as BT
    from drape_b200 import scenes as S
    b = BT.BatchSolver(0)
    for sc in S.batch_tubes(64)[:args.batch_garments]:
        b.add(sc)
    b.build()
    for g in range(b.size()[0]):
        b.set_phase(g, 0)
    for _ in range(args.batch_frames):
        b.step(1.0 / 60.0, 1, 2)
    G, N, B = b.size()
    print(json.dumps({"case": "batch", "garments": G, "particles": N, "block_slots": B, "frames": args.batch_frames,
                      "profile": b.profile_read()}))
    return 0


def cpu_baseline(workload: str):
    """The reference CPU path on this host's cores (reference_drape): one whole drape of the workload's own start
    state to rest, timed whole."""
    r = reference_drape(workload, 1, 0)
    sample = (f"one whole drape of the workload's own start state to rest ({r['frames']} frames, settled "
              f"{r['settled']}) on {r['threads']} host threads ({r['cpu']}, {r['host_cpus']} logical CPUs), "
              f"timed whole")
    return {"value": r["seconds"], "unit": "s", "cores": r["threads"], "kind": "port", "sample": sample,
            "frames": r["frames"], "pcg_iters_per_newton": r["cg_iterations"] / max(1, r["newton_iterations"])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="tube60k")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (0: same as --steps)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner leg")
    ap.add_argument("--refresh-every", type=int, default=1,
                    help="learned leg: run the network every this many Newton iterations")
    ap.add_argument("--no-deviation", action="store_true", help="skip the deviation-from-the-oracle leg")
    ap.add_argument("--pcg-variant", type=int, choices=[0, 1, 2, 3], default=0,
                    help="block-Jacobi PCG form: 0 the reference's order (resident rows where the scene fits), "
                         "1 pipelined (one grid exchange an iteration), 2 Chronopoulos-Gear (one reduction and one "
                         "plain barrier), 3 the reference's order on the 1024-thread kernel")
    ap.add_argument("--batch-garments", type=int, default=64, help="garments of the batched leg (0: skip it)")
    ap.add_argument("--profile-case", choices=["spmv", "batch", "bake", "drape", "drape_learned", "learned",
                                               "learned_inference"],
                    default=None,
                    help="run one small case for a profiler capture instead of the benchmark")
    ap.add_argument("--spmv-tiles", type=int, default=12)
    ap.add_argument("--batch-frames", type=int, default=6)
    ap.add_argument("--clock-period-ms", type=int, default=200, help="nvidia-smi clock sampling period")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_case:
        return run_profile_case(args)

    import torch
    from drape_b200 import cuda as CU

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        dist = None

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    scene = make_scene(args.workload)
    gid = scene.garments[0].id
    solver = CU.CudaSolver(local)
    solver.set_pcg_variant(args.pcg_variant)
    solver.build(scene)
    st = solver.structure()
    sizes = dict(n=len(st["diag_slot"]), B=len(st["col_index"]), S=len(st["stretch_v"]), H=len(st["hinge_v"]),
                 K=len(st["seam_ab"]))
    init = solver.snapshot()
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    base32 = np.ascontiguousarray(init["positions"], np.float32)
    seed_positions = [seeded_positions(base32, k) for k in range(SEEDS)]

    def one_drape(seed):
        snap = dict(init)
        snap["positions"] = seed_positions[seed]
        solver.restore(snap)
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # evict the L2 between drapes
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        res = solver.drape_to_rest([gid])
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end) / 1000.0, res

    for w in range(args.warmup):
        one_drape(w % SEEDS)

    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    gpu_id = gpu_uuid if gpu_uuid.startswith("GPU-") else "GPU-" + gpu_uuid
    # The timed drapes run the production path: profiling off, so every frame is one CUDA graph launch (kernel
    # events disable the frame graphs, and a drape launched kernel by kernel exposes host-side gaps between launches:
    # its device time per frame then varies with the host while the kernels' own time does not).
    solver.reset_counters()
    solver.profile(False)
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_id, args.clock_period_ms)
    times, results, per_drape = [], [], []
    last = solver.counters()
    for k in range(args.steps):
        t, res = one_drape(k % SEEDS)
        times.append(t)
        results.append(res)
        c = solver.counters()  # host read after the drape's end event, outside the timed events
        per_drape.append({"newton": c.newton_iterations - last.newton_iterations,
                          "cg": c.cg_iterations - last.cg_iterations,
                          "halvings": c.line_search_halvings - last.line_search_halvings})
        last = c
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    counters = solver.counters()
    cg_hist = solver.cg_history()
    settle_s = statistics.mean(times)
    value = max_over_ranks(settle_s)
    drapes = len(times)

    # Roofline of the dominant kernel (k_solve: persistent PCG + FP64 line search), from one more drape of the
    # workload's own start state outside the timed region with events around k_solve only.
    ab = algorithmic_bytes(sizes)
    solver.profile(True, solve_only=True)
    one_drape(0)
    prof = solver.profile_read()
    solver.profile(False)
    solve_ms = prof["milliseconds"]["k_solve"]
    solve_launches = max(1, prof["launches"]["k_solve"])
    solve_bytes = prof["cg_iterations"] * ab["pcg_iter"] + prof["energy_evaluations"] * ab["energy"]
    achieved = solve_bytes / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    peak, peak_kind = measured_peaks()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "k_solve_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            t = json.load(f)
        if t.get("workload") == args.workload and t.get("kernel") == ("k_solve_rows" if solver.solve_threads() == 512
                                                                      else "k_solve"):
            traffic = t.get("dram_bytes_per_launch")
    # Kernel shares from one more drape (the workload's own start state) with every kernel timed, outside the timed
    # region (events around every launch cost about 6 % of the frame time).
    solver.profile(True)
    _, share_res = one_drape(0)
    share_prof = solver.profile_read()
    solver.profile(False)
    # Kernels launched in the timed region: the profiled drape's launches per frame (k_advance_clock rides in
    # k_finish's events, so it is not counted) times the frames of the timed drapes.
    launches_timed = sum(share_prof["launches"].values()) / max(1, share_res.frames_run) * \
        sum(r.frames_run for r in results)
    total_ms = sum(share_prof["milliseconds"].values())
    # The bound that k_solve actually meets: its matrix (36 B a block slot) lives in shared memory and L2, so its time
    # per PCG iteration is set by the grid-wide exchanges. The PCG loop's own device time (%globaltimer, block 0) per
    # iteration is set beside the measured floor of the same exchanges on the same grid with no other work.
    pcg_us = counters.pcg_nanoseconds / 1000.0 / max(1, counters.cg_iterations)
    solve_threads = solver.solve_threads()
    floor_mode = {0: 0, 3: 0, 1: 2, 2: 1}[args.pcg_variant]
    floor_us = statistics.median(CU.reduction_floor(local, floor_mode + (4 if solve_threads == 512 else 0), 4000)
                                 for _ in range(3))
    latency = {"kernel": ("k_solve_rows" if solve_threads == 512 else "k_solve") + " PCG loop",
               "solve_threads": solve_threads, "us_per_pcg_iteration": pcg_us, "floor_us": floor_us,
               "floor": {0: "two FP64 grid reductions per iteration (reference-order PCG)",
                         2: "one three-value FP64 grid reduction per iteration (pipelined PCG)",
                         1: "one three-value FP64 grid reduction and one plain barrier per iteration "
                            "(Chronopoulos-Gear PCG)"}[floor_mode],
               "frac_of_floor": floor_us / pcg_us if pcg_us else None,
               "onchip_bytes_per_iteration": ab["pcg_iter"],
               "onchip_gbs": ab["pcg_iter"] / (pcg_us * 1e-6) / 1e9 if pcg_us else None,
               "note": f"floor = drape_cuda_reduction_floor on the solve's grid (one {solve_threads}-thread block per "
                       "SM), "
                       "median of 3 x 4000 rounds; us_per_pcg_iteration = in-kernel PCG time / PCG iterations over "
                       "the timed drapes (CG init amortised); onchip_gbs = the iteration's algorithmic bytes over its "
                       "time, served from shared memory and L2"}
    roofline = {"bound": "hbm", "kernel": "k_solve", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if peak else None, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": solve_bytes / solve_launches,
                "avg_launch_ms": solve_ms / solve_launches,
                "bound_note": "HBM is not what limits k_solve: its DRAM traffic is a small part of its algorithmic "
                              "bytes (the matrix sits in shared memory and L2); the limit is grid-exchange latency, "
                              "see the line's k_solve_latency object",
                "kernel_share": {k: (v / total_ms if total_ms else 0.0) for k, v in share_prof["milliseconds"].items()},
                "kernel_share_sample": "one extra drape of the workload's own start state, every kernel timed"}

    # End to end through the C ABI with host buffers: build from host arrays (H2D), drape, read positions (D2H), for
    # the same seeded start states.
    e2e_steps = args.e2e_steps or args.steps
    e2e_times, e2e_build, h2d, d2h, e2e_frames = [], [], [], [], []
    garment = scene.garments[0]
    own = garment.initial_positions
    for k in range(e2e_steps):
        garment.initial_positions = seed_positions[k % SEEDS].astype(np.float64)
        torch.cuda.synchronize()
        b0 = solver.transfer_bytes()
        t0 = time.perf_counter()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        solver.build(scene)
        e2e_build.append(time.perf_counter() - t0)
        e2e_frames.append(int(solver.drape_to_rest([gid]).frames_run))
        out = np.empty((sizes["n"], 3), np.float32)
        solver.read_positions(out)
        end.record(stream)
        end.synchronize()
        wall = time.perf_counter() - t0
        e2e_times.append(max(wall, start.elapsed_time(end) / 1000.0))
        b1 = solver.transfer_bytes()
        h2d.append(b1[0] - b0[0])
        d2h.append(b1[1] - b0[1])
    garment.initial_positions = own
    e2e_value = max_over_ranks(statistics.mean(e2e_times))
    solver.restore(init)
    solver.drape_to_rest([gid])  # the block-Jacobi drape's final shape from the workload's own start state

    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1000.0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "precond": "block-Jacobi",
                   "pcg": {0: "reference order (two grid reductions per iteration)",
                           3: "reference order (two grid reductions per iteration)",
                           1: "pipelined (one grid reduction per iteration)",
                           2: "Chronopoulos-Gear (one grid reduction and one plain barrier per iteration)"}[
                               args.pcg_variant] + (", resident rows (512-thread blocks)" if solve_threads == 512
                                                    else ", 1024-thread blocks"),
                   "start_states": SEED_DESC,
                   "precision": "FP32 blocks/SpMV/vectors, FP64 dots, FP64 energy/slope/line search",
                   "l2": "256 MB buffer written between timed drapes (L2 flushed)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "s", "h2d_bytes_per_step": int(sum(h2d) / e2e_steps),
                "d2h_bytes_per_step": int(sum(d2h) / e2e_steps), "drapes": len(e2e_times),
                "frames_per_step": e2e_frames, "frames_mean": float(np.mean(e2e_frames)),
                "s_per_step": [round(t, 4) for t in e2e_times],
                "build_s_per_step": [round(t, 4) for t in e2e_build],
                "note": "mean seconds per drape (one drape per step, the same start states as the timed steps); "
                        "bytes per step"},
        "roofline": roofline,
        "k_solve_latency": latency,
        "clocks": clocks,
        "gpu_launches": int(launches_timed),
        "drape": {"drapes_timed": drapes,
                  "frames_per_step": [int(r.frames_run) for r in results],
                  "settled_per_step": [bool(r.settled) for r in results],
                  "settle_s_per_step": [round(float(t), 4) for t in times],
                  "ms_per_frame_per_step": [round(1000.0 * t / max(1, r.frames_run), 3)
                                            for t, r in zip(times, results)],
                  "work_per_step": per_drape,
                  "settle_s_median": float(np.median(times)),
                  "frames_mean": float(np.mean([r.frames_run for r in results])),
                  "assembly_seconds": float(results[-1].assembly_seconds),
                  "retries": int(sum(r.retries for r in results)),
                  "newton_iterations_per_drape": counters.newton_iterations / drapes,
                  "ms_per_frame": 1000.0 * sum(times) / max(1, sum(r.frames_run for r in results)),
                  "drapes_per_s": world / value if value else None},
        "pcg_iters_per_newton": {"mean": float(np.mean(cg_hist)) if len(cg_hist) else None,
                                 "p50": float(np.percentile(cg_hist, 50)) if len(cg_hist) else None,
                                 "p95": float(np.percentile(cg_hist, 95)) if len(cg_hist) else None,
                                 "cap": 50},
        "sizes": sizes,
    }
    jac_final = solver.positions().astype(np.float64)
    if rank == 0 and not args.no_deviation:
        line["deviation"] = deviation_leg(CU, local, jac_final if args.workload == "tube60k" else None,
                                          args.pcg_variant)
    if not args.no_learned:
        line["precond"] = precond_leg(CU, local, args, flush, max_over_ranks)
    peak, _ = measured_peaks()
    solver.restore(init)
    line["spmv"] = spmv_leg(CU, solver, peak)
    big = spmv_leg(CU, solver, peak, tiles=24)  # twice the matrix (568 MB), the HBM-resident regime of the batch
    line["spmv"]["larger_matrix"] = {k: big[k] for k in ("matrix_mb", "ms_per_launch", "achieved", "frac",
                                                          "max_rel_error_vs_host")}
    if args.batch_garments > 0:
        line["batch"] = batch_leg(args, local, world, rank, max_over_ranks, peak)
    if rank == 0:
        line["bake"] = bake_leg(peak)
        line["mesh"] = mesh_leg()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    if rank == 0:
        print(json.dumps(line))
    solver.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
