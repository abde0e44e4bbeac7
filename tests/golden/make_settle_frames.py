"""Generates tests/golden/settle_frames.json: the reference CPU path (the oracle's faithful restatement of CpuSolver,
one thread) draped to rest on each benchmark workload with the drape runner's criterion.

For each workload it records the frames to settle, the total wall time of the drape on the machine that ran this
script, and the wall time of the first `sample` frames. The benchmark's reference arm times those same first frames
on its own host and scales the total by the ratio, so that the full CPU drape need not be rerun every time.

Run: python tests/golden/make_settle_frames.py [tube10k] [tube60k]
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "drape-2_b200"))

import oracle as O  # noqa: E402
from drape_b200 import scenes as S  # noqa: E402
from drape_b200 import session as SS  # noqa: E402

OUT = os.path.join(HERE, "settle_frames.json")
SAMPLE = {"tube10k": 20, "tube60k": 5}
MAKERS = {"tube10k": S.tube_10k, "tube60k": S.tube_60k}


def run(workload: str) -> dict:
    scene = MAKERS[workload]()
    o = O.OracleSolver()
    o.build(scene)
    sess = SS.DrapeSession(o, [scene.garments[0].id])
    t0 = time.perf_counter()
    sample_s = None
    frames = 0
    while not sess.finished():
        sess.advance()
        frames += 1
        if frames == SAMPLE[workload]:
            sample_s = time.perf_counter() - t0
    total = time.perf_counter() - t0
    c = o.counters()
    r = sess.result
    return {"frames": r.frames_run, "settled": r.settled, "simulated_seconds": r.simulated_seconds,
            "assembly_seconds": r.assembly_seconds, "retries": r.retries, "total_seconds": total,
            "sample_frames": SAMPLE[workload], "sample_seconds": sample_s,
            "newton_iterations": c.newton_iterations, "cg_iterations": c.cg_iterations,
            "host": platform.processor() or platform.machine()}


def main():
    names = sys.argv[1:] or sorted(MAKERS)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for name in names:
        data[name] = run(name)
        print(name, data[name], flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
