"""Training data and training for the learned preconditioner, all on the GPU.

Samples are Newton systems logged from drapes of seeded tube variants (panel sizes +-20 %, body radii +-15 %): every
`every` frames the solver's next system is captured (block Hessian, contact flags) with seeded Gaussian probe
vectors for the Kaporin objective. ``train`` runs Adam on the device (drape_precond_train) and returns the losses;
``python -m drape_b200.train --out weights.npy`` writes trained parameters.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import cuda, learned, scenes


def collect(precond: learned.LearnedPreconditioner, seeds, n_particles: int = 6000, frames: int = 120,
            every: int = 15, probes: int = 4, device: int = 0, field_n: int = 96) -> int:
    """Drapes each seeded variant for `frames` frames and adds a sample every `every` frames, each with `probes`
    seeded standard-normal probe vectors (the Kaporin objective's). Returns the count."""
    added = 0
    for seed in seeds:
        scene = scenes.tube_variant(int(seed), n_particles, field_n=field_n)
        s = cuda.CudaSolver(device)
        s.build(scene)
        gid = scene.garments[0].id
        rng = np.random.default_rng(1000 + int(seed))
        for f in range(frames):
            if f == 30:
                s.set_phase(gid, 1)  # settle after half a second of assembly
            if f % every == every - 1:
                sysm = s.capture_system(1.0 / 60.0)
                n = len(sysm["diag_slot"])
                res = [rng.standard_normal((n, 3)).astype(np.float32) for _ in range(probes)]
                precond.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"], np.zeros(n, np.uint8),
                                   sysm["active"], np.stack(res))
                added += 1
            s.step(1.0 / 60.0, 1, 2)
        s.close()
    return added


def collect_c4(precond: learned.LearnedPreconditioner, count: int = 200, n_min: int = 5000, n_max: int = 40000,
               seed: int = 4, probes: int = 4, device: int = 0, field_n: int = 128) -> dict:
    """The learned-preconditioner training set of the workload definition: `count` seeded tube variants (panel sizes
    +-20 %, torso and arm radii +-15 %; drape_b200.scenes.tube_variant) with particle counts log-uniform in
    [n_min, n_max], each draped by the block-Jacobi solver (Assembling for 30 frames, then Settling) and logged once,
    at a seeded frame in 20-119, as its Newton system (block Hessian, contact flags) with `probes` seeded Gaussian probe
    vectors. One system per variant keeps the device-side training workspace (about 1 KB per block slot) near 60 GB
    for 200 variants. Returns the variant seeds, sizes and frames."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).round().astype(int)
    frames = rng.integers(20, 120, count)
    seeds = [2000 + k for k in range(count)]
    for k in range(count):
        scene = scenes.tube_variant(seeds[k], int(sizes[k]), field_n=field_n)
        s = cuda.CudaSolver(device)
        s.build(scene)
        gid = scene.garments[0].id
        s.set_phase(gid, 0)
        for f in range(int(frames[k])):
            if f == 30:
                s.set_phase(gid, 1)
            s.step(1.0 / 60.0, 1, 2)
        sysm = s.capture_system(1.0 / 60.0)
        n = len(sysm["diag_slot"])
        prng = np.random.default_rng(10_000 + k)
        res = np.stack([prng.standard_normal((n, 3)).astype(np.float32) for _ in range(probes)])
        precond.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"], np.zeros(n, np.uint8),
                           sysm["active"], res)
        s.close()
    return {"seeds": seeds, "sizes": sizes.tolist(), "frames": frames.tolist()}


def train(precond: learned.LearnedPreconditioner, steps: int = 1500, lr: float = 1e-3, batch: int = 4,
          seed: int = 0) -> np.ndarray:
    return precond.train(steps, lr=lr, batch=batch, seed=seed)


def capture_along_drape(scene, frames: int = 120, every: int = 10, device: int = 0):
    """Newton systems captured every `every` frames of a block-Jacobi drape (Settling from frame 30)."""
    s = cuda.CudaSolver(device)
    s.build(scene)
    gid = scene.garments[0].id
    out = []
    for f in range(frames):
        if f == 30:
            s.set_phase(gid, 1)
        if f % every == every - 1:
            out.append(s.capture_system(1.0 / 60.0))
        s.step(1.0 / 60.0, 1, 2)
    s.close()
    return out


def ablation(params, systems, tolerance: float = 1e-2, max_iterations: int = 2000, device: int = 0) -> dict:
    """PCG iterations of block-Jacobi and of the learned preconditioner on the same systems (drape_precond_pcg, right
    side -grad, no contact filter). Returns the per-system counts and their means."""
    ev = learned.LearnedPreconditioner(device, params)
    jac, lrn = [], []
    for sysm in systems:
        n = len(sysm["diag_slot"])
        sid = ev.add_sample(sysm["row_start"], sysm["col_index"], sysm["blocks"], np.zeros(n, np.uint8),
                            sysm["active"], (-sysm["grad"])[None])
        jac.append(ev.pcg(sid, 0, False, max_iterations, tolerance)[0])
        lrn.append(ev.pcg(sid, 0, True, max_iterations, tolerance)[0])
        ev.clear_samples()
    ev.close()
    return dict(jacobi=jac, learned=lrn, jacobi_mean=float(np.mean(jac)), learned_mean=float(np.mean(lrn)),
                ratio=float(np.mean(jac) / max(np.mean(lrn), 1e-9)), tolerance=tolerance)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="weights.npy")
    ap.add_argument("--variants", type=int, default=6)
    ap.add_argument("--n", type=int, default=6000)
    ap.add_argument("--frames", type=int, default=120)
    ap.add_argument("--every", type=int, default=15)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--sizes", default="", help="comma-separated particle counts cycled over the variants")
    ap.add_argument("--ablate", default="",
                    help="evaluate these weights (.npy) against block-Jacobi on held-out systems and print JSON")
    ap.add_argument("--c4", type=int, default=0,
                    help="train on this many seeded variants of 5k-40k particles, one system each (collect_c4)")
    args = ap.parse_args()
    if args.ablate:
        import json
        params = np.load(args.ablate)
        out = []
        cases = [(f"variant {sd}, {n} particles", scenes.tube_variant(sd, n)) for sd, n in
                 ((7, 5000), (8, 10000), (9, 20000), (10, 40000))] + [("tube60k (bench workload)", scenes.tube_60k())]
        for name, scene in cases:
            systems = capture_along_drape(scene, frames=120, every=20)
            for tol in (1e-2, 1e-4):
                r = ablation(params, systems, tolerance=tol)
                out.append({"system": name, "tolerance": tol, "systems": len(systems), "jacobi": r["jacobi_mean"],
                            "learned": r["learned_mean"], "ratio": r["ratio"]})
                print(json.dumps(out[-1]), flush=True)
        return
    p = learned.LearnedPreconditioner(0, learned.init_params(args.seed))
    t0 = time.perf_counter()
    if args.c4:
        info = collect_c4(p, args.c4)
        t1 = time.perf_counter()
        losses = train(p, args.steps, args.lr, args.batch, args.seed)
        t2 = time.perf_counter()
        np.save(args.out, p.params())
        k = max(1, len(losses) // 10)
        print(f"c4: {args.c4} variants ({min(info['sizes'])}-{max(info['sizes'])} particles) in {t1 - t0:.1f} s; "
              f"{args.steps} Adam steps in {t2 - t1:.1f} s; loss {np.mean(losses[:k]):.4f} -> {np.mean(losses[-k:]):.4f}")
        return
    sizes = [int(x) for x in args.sizes.split(",") if x] or [args.n]
    count = 0
    for k in range(args.variants):
        count += collect(p, [100 + k], sizes[k % len(sizes)], args.frames, args.every)
    t1 = time.perf_counter()
    losses = train(p, args.steps, args.lr, args.batch, args.seed)
    t2 = time.perf_counter()
    np.save(args.out, p.params())
    k = max(1, len(losses) // 10)
    print(f"samples {count} in {t1 - t0:.1f} s; {args.steps} Adam steps in {t2 - t1:.1f} s; "
          f"loss {np.mean(losses[:k]):.4f} -> {np.mean(losses[-k:]):.4f}")


if __name__ == "__main__":
    main()
