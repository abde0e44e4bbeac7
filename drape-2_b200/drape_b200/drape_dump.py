"""drape_dump: drapes one workload to rest through the GPU/CPU solver switch and writes the garment as OBJ.

Restates the reference tool (tools/drape_dump/main.cpp:61-104: build a scene, drapeToRest, print one summary line,
exit 0 when settled) with the backend choice the application's toolbar makes (sim_controller.hpp:25,
apps/drape/main_window.cpp:91): `--backend cuda` drapes on this library's CUDA solver and, through SimController,
falls back to the CPU backend when the GPU cannot be used or fails mid-drape; `--backend cpu` drapes on the CPU
backend. The CPU backend is the caller's Solver class, named with `--cpu-solver module:attribute` (the reference's
CpuSolver in the application); without it, a GPU failure ends the drape as Failed.

  python -m drape_b200.drape_dump --workload tube10k [--backend cuda|cpu] [--cpu-solver mod:Cls] [--out tube.obj]
"""
from __future__ import annotations

import argparse
import importlib
import sys

import numpy as np

from . import controller as SC
from . import scenes as S
from . import session as SS

WORKLOADS = {
    "patch": lambda: S.Scene([S.centred_sheet(0.04, 0.01, 0.2)], S.sphere_field()),  # 25 particles onto the sphere
    "sheet": S.sheet_on_sphere, "tube10k": S.tube_10k, "tube60k": S.tube_60k,
}


def load_attribute(spec: str):
    module, _, attr = spec.partition(":")
    if not module or not attr:
        raise ValueError(f"--cpu-solver wants module:attribute, got '{spec}'")
    return getattr(importlib.import_module(module), attr)


def write_obj(path: str, positions: np.ndarray, triangles: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("o garment\n")
        for p in positions:
            f.write(f"v {p[0]:.6f} {p[1]:.6f} {p[2]:.6f}\n")
        for t in triangles:
            f.write(f"f {t[0] + 1} {t[1] + 1} {t[2] + 1}\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="drape_dump")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="tube10k")
    ap.add_argument("--backend", choices=[SC.CUDA, SC.CPU], default=SC.CUDA)
    ap.add_argument("--cpu-solver", default=None, help="module:attribute of the CPU Solver class")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="OBJ file for the draped garment")
    ap.add_argument("--timeout", type=float, default=3600.0, help="wall seconds to wait for the drape")
    args = ap.parse_args(argv)
    try:
        cpu = load_attribute(args.cpu_solver) if args.cpu_solver else None
        scene = WORKLOADS[args.workload]()
        config = SC.SimConfig(scene=lambda: scene, garments=tuple(g.id for g in scene.garments), backend=args.backend)
        ctl = SC.SimController(config, SC.cuda_factory(args.device, cpu))
        try:
            ctl.set_running(True)
            done = (SS.STATE_SETTLED, SS.STATE_FAILED, SS.STATE_TIMED_OUT)
            st = ctl.wait(lambda s: s.revision > 0 and s.state in done and not s.running, timeout=args.timeout)
            frame = ctl.exchange.latest()
            solver = ctl._solver
            stats = solver.stats() if solver is not None else None
        finally:
            ctl.close()
    except Exception as e:  # noqa: BLE001
        print(f"drape_dump: {e}", file=sys.stderr)
        return 1
    if args.out and frame is not None:
        offset, tris = 0, []
        for g in scene.garments:
            tris.append(np.asarray(g.triangles, np.int64) + offset)
            offset += g.vertex_count
        write_obj(args.out, frame.positions, np.concatenate(tris))
    settled = st.state == SS.STATE_SETTLED
    failed = st.state == SS.STATE_FAILED
    gap = stats.max_seam_gap if stats is not None else float("nan")
    pen = max(0.0, stats.max_body_penetration) if stats is not None else float("nan")
    print(f"settled={int(settled)} failed={int(failed)} seconds={st.simulated_seconds:.2f} frames={st.frames} "
          f"seam_gap_mm={gap * 1000.0:.2f} penetration_mm={pen * 1000.0:.2f} particles={st.particles} "
          f"backend={st.backend}" + (f" note=\"{st.message}\"" if st.message else ""))
    return 0 if settled and not failed else 1


if __name__ == "__main__":
    sys.exit(main())
