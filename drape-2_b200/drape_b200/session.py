"""The drape runner over any object with the Solver interface (step, stats, snapshot, restore, set_phase).

Restates DrapeSession (libs/sim/src/drape_session.cpp:12-95, libs/sim/include/drape/sim/drape_session.hpp) and
drapeToRest (libs/sim/src/drape_runner.cpp:7-11): Assembling -> Settling -> Settled, the stability guard (non-finite
state or kinetic energy rising for energyRiseFrames frames -> restore the last snapshot and double the substeps, at
most maxRetries times), a snapshot every snapshotEvery kept frames, and the timeouts. The CUDA library carries its own
C++ copy of this loop with device-side snapshots (drape_cuda_drape_to_rest); this one drives the CPU oracle and
scripted test solvers.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

ASSEMBLING, SETTLING = 0, 1
STATE_ASSEMBLING, STATE_SETTLING, STATE_SETTLED, STATE_FAILED, STATE_TIMED_OUT = range(5)
FAILURE_MESSAGE = "Drape couldn't settle this garment. Try Draft quality or a different fabric."
_TIME_EPS = 1e-9


@dataclass
class DrapeOptions:
    substeps: int = 1
    iterations: int = 2
    frame_dt: float = 1.0 / 60.0
    max_assembly_seconds: float = 3.0
    seam_gap_done: float = 0.001
    settle_rms_speed: float = 0.002
    settle_hold_frames: int = 60
    max_sim_seconds: float = 20.0
    snapshot_every: int = 30
    max_retries: int = 3
    energy_rise_frames: int = 60
    frames_per_wait: int = 10  # device frames per host wait in the C runner (same outcome for every value)

    def to_c(self):
        from .scene import drape_drape_options
        return drape_drape_options(self.substeps, self.iterations, self.frame_dt, self.max_assembly_seconds,
                                   self.seam_gap_done, self.settle_rms_speed, self.settle_hold_frames,
                                   self.max_sim_seconds, self.snapshot_every, self.max_retries,
                                   self.energy_rise_frames, self.frames_per_wait)


@dataclass
class DrapeResult:
    settled: bool = False
    failed: bool = False
    message: str = ""
    simulated_seconds: float = 0.0
    retries: int = 0
    frames_run: int = 0
    assembly_end_seam_gap: float = 0.0
    assembly_seconds: float = 0.0


class DrapeSession:
    def __init__(self, solver, garments, options: DrapeOptions = DrapeOptions()):
        self.s, self.garments, self.o = solver, list(garments), options
        self.result = DrapeResult()
        self.state, self.phase = STATE_ASSEMBLING, ASSEMBLING
        self.time = self.phase_time = 0.0
        self.substeps = options.substeps
        self.still = self.rise = self.kept = 0
        self.last_energy = math.inf
        self._set_all(ASSEMBLING)
        self.saved = (solver.snapshot(), 0.0, ASSEMBLING, 0.0)

    def _set_all(self, p):
        for g in self.garments:
            self.s.set_phase(g, p)

    def _reset_counters(self):
        self.still = self.rise = 0
        self.last_energy = math.inf

    def finished(self) -> bool:
        return self.state in (STATE_SETTLED, STATE_FAILED, STATE_TIMED_OUT)

    def advance(self) -> int:
        o, r = self.o, self.result
        if self.finished():
            return self.state
        if self.time >= o.max_sim_seconds - _TIME_EPS:
            r.simulated_seconds = self.time
            self.state = STATE_TIMED_OUT
            return self.state
        self.s.step(o.frame_dt, self.substeps, o.iterations)
        r.frames_run += 1
        self.kept += 1
        self.time += o.frame_dt
        self.phase_time += o.frame_dt
        st = self.s.stats()
        self.rise = self.rise + 1 if st.kinetic_energy > self.last_energy else 0
        self.last_energy = st.kinetic_energy
        if st.has_non_finite or self.rise >= o.energy_rise_frames:
            r.retries += 1
            if r.retries > o.max_retries:
                r.retries = o.max_retries
                r.failed = True
                r.message = FAILURE_MESSAGE
                r.simulated_seconds = self.time
                self.state = STATE_FAILED
                return self.state
            snap, t, ph, pt = self.saved
            self.s.restore(snap)
            self.time, self.phase, self.phase_time = t, ph, pt
            self.kept = int(t / o.frame_dt + 0.5)
            self.substeps *= 2
            self._reset_counters()
            self.state = STATE_ASSEMBLING if self.phase == ASSEMBLING else STATE_SETTLING
            return self.state
        if self.phase == ASSEMBLING:
            if st.max_seam_gap < o.seam_gap_done or self.phase_time >= o.max_assembly_seconds - _TIME_EPS:
                r.assembly_end_seam_gap = st.max_seam_gap
                r.assembly_seconds = self.time
                self.phase = SETTLING
                self._set_all(SETTLING)
                self.phase_time = 0.0
                self._reset_counters()
        else:
            self.still = self.still + 1 if st.rms_speed < o.settle_rms_speed else 0
            if self.still >= o.settle_hold_frames:
                r.settled = True
                r.simulated_seconds = self.time
                self.state = STATE_SETTLED
                return self.state
        if self.kept % o.snapshot_every == 0:
            self.saved = (self.s.snapshot(), self.time, self.phase, self.phase_time)
        if self.time >= o.max_sim_seconds - _TIME_EPS:
            r.simulated_seconds = self.time
            self.state = STATE_TIMED_OUT
            return self.state
        self.state = STATE_ASSEMBLING if self.phase == ASSEMBLING else STATE_SETTLING
        return self.state


def drape_to_rest(solver, garments, options: DrapeOptions = DrapeOptions()) -> DrapeResult:
    session = DrapeSession(solver, garments, options)
    while not session.finished():
        session.advance()
    return session.result
