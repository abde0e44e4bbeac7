#!/usr/bin/env python
"""Benchmark of the cloth solver's Newton-step hot path on B200: drape settle time.

One step = one drape of the seamed-tube workload to rest, run by the solver's drape runner (DrapeSession semantics,
libs/sim/src/drape_session.cpp:32-95: Assembling until the seams close, then Settling until the RMS speed stays below
2 mm/s for 60 frames). The metric is the wall time to settle; PCG iterations per Newton step are reported beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference] [--workload tube60k|tube10k]

--impl cuda (default): the CUDA library through its C ABI, inputs resident in HBM (value) and through the full
  host-buffer path (e2e: build from host arrays, drape, read positions back). For N > 1 every rank drapes its own
  replica (one drape does not shard); value is the slowest rank's settle time.
--impl reference: the reference solver's CPU algorithm (the oracle's restatement of CpuSolver, single-threaded like
  the reference) timed on a bounded sample of frames of the same workload, extrapolated to the frames the reference
  path needs to settle (tests/golden/settle_frames.json, made by tests/golden/make_settle_frames.py).
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

    def __init__(self, gpu_id: str):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", gpu_id], stdout=self.file, stderr=subprocess.DEVNULL)
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
        sm, smax, reasons = [], [], set()
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
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_settle_seconds(workload: str, repeats: int):
    """The reference CPU path's settle time on this host: the first `sample` frames of the drape are timed here
    (`repeats` times, the fastest kept), and the full drape's wall time recorded by tests/golden/make_settle_frames.py
    on its machine is scaled by the ratio of the two sample times. Returns (seconds, description, fixture)."""
    import oracle as O
    from drape_b200 import session as SS
    with open(SETTLE_FIXTURE) as f:
        fx = json.load(f)[workload]
    scene = make_scene(workload)
    sample = int(fx["sample_frames"])
    best = None
    for _ in range(max(1, repeats)):
        o = O.OracleSolver()
        o.build(scene)
        sess = SS.DrapeSession(o, [scene.garments[0].id])
        t0 = time.perf_counter()
        for _ in range(sample):
            sess.advance()
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    value = float(fx["total_seconds"]) * best / float(fx["sample_seconds"])
    desc = (f"first {sample} frames of the drape timed on this host ({best:.2f} s, one thread); the full drape "
            f"({fx['frames']} frames to settle, {fx['total_seconds']:.1f} s where the fixture was made, sample "
            f"{fx['sample_seconds']:.2f} s) scaled by the sample ratio")
    return value, desc, fx


def run_reference(args):
    """The reference CPU path (oracle restatement of CpuSolver, float state, double solve, one thread)."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    value, desc, fx = reference_settle_seconds(args.workload, args.warmup + args.steps)
    line = {
        "metric": METRIC, "value": value, "unit": "s", "impl": "reference", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1000.0, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"],
                   "solver": "CpuSolver restatement (float particle state, double solve), block-Jacobi PCG"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "frames_to_settle": int(fx["frames"]),
        "pcg_iters_per_newton": {"mean": fx["cg_iterations"] / max(1, fx["newton_iterations"]), "cap": 50},
    }
    print(json.dumps(line))
    return 0


def cpu_baseline(workload: str):
    try:
        value, desc, _ = reference_settle_seconds(workload, 1)
    except (OSError, KeyError) as e:
        return {"value": None, "unit": "s", "cores": 1, "kind": "port", "sample": f"no settle fixture: {e}"}
    return {"value": value, "unit": "s", "cores": 1, "kind": "port", "sample": desc}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="tube60k")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (0: same as --steps)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

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
    solver.build(scene)
    st = solver.structure()
    sizes = dict(n=len(st["diag_slot"]), B=len(st["col_index"]), S=len(st["stretch_v"]), H=len(st["hinge_v"]),
                 K=len(st["seam_ab"]))
    init = solver.snapshot()
    stream = torch.cuda.ExternalStream(solver.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > 126 MB L2

    def one_drape():
        solver.restore(init)
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # evict the L2 between drapes
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        res = solver.drape_to_rest([gid])
        end.record(stream)
        end.synchronize()
        return start.elapsed_time(end) / 1000.0, res

    for _ in range(args.warmup):
        one_drape()

    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    gpu_id = gpu_uuid if gpu_uuid.startswith("GPU-") else "GPU-" + gpu_uuid
    solver.reset_counters()
    solver.profile(True)
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_id)
    times, results = [], []
    for _ in range(args.steps):
        t, res = one_drape()
        times.append(t)
        results.append(res)
    barrier()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    prof = solver.profile_read()
    solver.profile(False)
    counters = solver.counters()
    cg_hist = solver.cg_history()
    settle_s = statistics.mean(times)
    value = max_over_ranks(settle_s)

    # Roofline of the dominant kernel (k_solve: persistent PCG + FP64 line search).
    ab = algorithmic_bytes(sizes)
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
        if t.get("workload") == args.workload:
            traffic = t.get("dram_bytes_per_launch")
    total_ms = sum(prof["milliseconds"].values())
    roofline = {"bound": "hbm", "kernel": "k_solve", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if peak else None, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": solve_bytes / solve_launches,
                "avg_launch_ms": solve_ms / solve_launches,
                "kernel_share": {k: (v / total_ms if total_ms else 0.0) for k, v in prof["milliseconds"].items()}}

    # End to end through the C ABI with host buffers: build from host arrays (H2D), drape, read positions (D2H).
    e2e_steps = args.e2e_steps or args.steps
    e2e_times, h2d, d2h = [], [], []
    for _ in range(e2e_steps):
        torch.cuda.synchronize()
        b0 = solver.transfer_bytes()
        t0 = time.perf_counter()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        solver.build(scene)
        solver.drape_to_rest([gid])
        out = np.empty((sizes["n"], 3), np.float32)
        solver.read_positions(out)
        end.record(stream)
        end.synchronize()
        wall = time.perf_counter() - t0
        e2e_times.append(max(wall, start.elapsed_time(end) / 1000.0))
        b1 = solver.transfer_bytes()
        h2d.append(b1[0] - b0[0])
        d2h.append(b1[1] - b0[1])
    e2e_value = max_over_ranks(statistics.mean(e2e_times))

    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1000.0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload]["desc"], "precond": "block-Jacobi",
                   "precision": "FP32 blocks/SpMV/vectors, FP64 dots, FP64 energy/slope/line search",
                   "l2": "256 MB buffer written between timed drapes (L2 flushed)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "s", "h2d_bytes_per_step": int(statistics.mean(h2d)),
                "d2h_bytes_per_step": int(statistics.mean(d2h))},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": int(sum(prof["launches"].values())),
        "drape": {"frames": int(results[-1].frames_run), "settled": bool(results[-1].settled),
                  "simulated_seconds": float(results[-1].simulated_seconds),
                  "assembly_seconds": float(results[-1].assembly_seconds), "retries": int(results[-1].retries),
                  "newton_iterations_per_drape": counters.newton_iterations / args.steps,
                  "ms_per_frame": 1000.0 * statistics.mean(t / max(1, r.frames_run) for t, r in zip(times, results)),
                  "drapes_per_s": world / value if value else None},
        "pcg_iters_per_newton": {"mean": float(np.mean(cg_hist)) if len(cg_hist) else None,
                                 "p50": float(np.percentile(cg_hist, 50)) if len(cg_hist) else None,
                                 "p95": float(np.percentile(cg_hist, 95)) if len(cg_hist) else None,
                                 "cap": 50},
        "sizes": sizes,
    }
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
