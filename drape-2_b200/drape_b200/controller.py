"""The GPU/CPU solver switch as running code: the reference's SimController (libs/session/src/sim_controller.cpp)
over any Solver factory, with the CUDA library as the GPU backend.

SimController owns one drape at a time on a worker thread, like the reference (sim_controller.cpp:57-98):
  - rebuild (sim_controller.cpp:100-150): makes a solver for the configured backend and builds the scene; when the
    GPU backend cannot be created or built (CudaError, DRAPE_DEVICE_ERROR at the C ABI), it notes
    "GPU unavailable: <cause>; using CPU" and builds on the CPU backend instead;
  - stepFailed (sim_controller.cpp:152-176): when a frame throws on the GPU backend (a device fault mid-drape), it
    notes "GPU failed: <cause>; using CPU", switches the configuration to the CPU backend and restarts the drape there;
    on the CPU backend the drape ends Failed with the error's message;
  - publish (sim_controller.cpp:178-186): after every frame the latest positions go to a one-slot exchange that a
    reader polls (PositionExchange).
Once the GPU has failed, its note stays in the status of every later CPU drape.

The factory maps a backend name ("cuda" or "cpu") to a new Solver; `cuda_factory` supplies "cuda" from this library.
The CPU backend is the caller's: in the reference application it is CpuSolver (libs/sim/src/cpu_solver.cpp); this
library has no CPU solver of its own.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field, replace
from typing import Callable, Optional

import numpy as np

from . import session as SS

CUDA, CPU = "cuda", "cpu"


def cuda_factory(device: int = 0, cpu: Optional[Callable[[], object]] = None) -> Callable[[str], object]:
    """A SolverFactory: "cuda" makes a CudaSolver on `device`; "cpu" calls `cpu()` (the caller's CPU solver), and
    raises ValueError when none was given."""
    def make(backend: str):
        if backend == CUDA:
            from . import cuda
            return cuda.make_solver(CUDA, device)
        if backend == CPU:
            if cpu is None:
                raise ValueError("no CPU solver was given to the solver factory")
            return cpu()
        raise ValueError(f"unknown solver backend '{backend}'")
    return make


@dataclass
class SimConfig:
    """sim_controller.hpp:22-30: what to drape and on which backend. `scene` is a callable returning the scene to
    build (the reference builds its tee scene from body, quality and size), `garments` the garment ids to drape."""
    scene: Callable[[], object]
    garments: tuple
    backend: str = CUDA
    options: SS.DrapeOptions = field(default_factory=SS.DrapeOptions)


@dataclass
class SimStatus:
    state: int = SS.STATE_ASSEMBLING
    running: bool = False
    particles: int = 0
    fps: float = 0.0
    simulated_seconds: float = 0.0
    message: str = ""
    backend: str = CUDA
    gpu_available: bool = True
    revision: int = 0
    frames: int = 0


@dataclass
class PublishedFrame:
    revision: int
    frame: int
    positions: np.ndarray


class PositionExchange:
    """The latest published frame (one slot, replaced on publish)."""

    def __init__(self):
        self._lock = threading.Lock()
        self._frame: Optional[PublishedFrame] = None

    def publish(self, f: PublishedFrame) -> None:
        with self._lock:
            self._frame = f

    def latest(self) -> Optional[PublishedFrame]:
        with self._lock:
            return self._frame


class SimController:
    def __init__(self, config: SimConfig, factory: Callable[[str], object]):
        self.factory = factory
        self._config = config
        self._status = SimStatus(backend=config.backend)
        self.exchange = PositionExchange()
        self._cv = threading.Condition()
        self._stop = self._running = False
        self._rebuild_pending = True
        self._session: Optional[SS.DrapeSession] = None
        self._solver = None
        self._backend = config.backend
        self._gpu_note = ""
        self._revision = self._frame = 0
        self._frame_times: list = []
        self._thread = threading.Thread(target=self._loop, name="sim", daemon=True)
        self._thread.start()

    # ---- the controller's public interface (sim_controller.hpp:32-47) ----
    def set_running(self, running: bool) -> None:
        with self._cv:
            self._running = running
            self._cv.notify_all()

    def reset(self) -> None:
        with self._cv:
            self._rebuild_pending = True
            self._cv.notify_all()

    def configure(self, config: SimConfig) -> None:
        with self._cv:
            self._config = config
            self._rebuild_pending = True
            self._cv.notify_all()

    def status(self) -> SimStatus:
        with self._cv:
            return replace(self._status)

    def close(self) -> None:
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        self._thread.join()
        self._session = None
        self._close_solver()

    def wait(self, predicate: Callable[[SimStatus], bool], timeout: float = 60.0) -> SimStatus:
        """Blocks until predicate(status) holds (or `timeout` seconds pass) and returns the status."""
        end = time.monotonic() + timeout
        with self._cv:
            while not predicate(self._status) and time.monotonic() < end:
                self._cv.wait(timeout=min(0.05, max(0.0, end - time.monotonic())))
            return replace(self._status)

    # ---- the sim thread ----
    def _ready(self) -> bool:
        return self._stop or self._rebuild_pending or (
            self._running and self._session is not None and not self._session.finished())

    def _loop(self) -> None:
        while True:
            with self._cv:
                if not self._ready():
                    self._status.running = False
                    self._status.fps = 0.0
                    self._cv.notify_all()
                    while not self._ready():
                        self._cv.wait()
                if self._stop:
                    return
                self._status.running = True
                rebuild = self._rebuild_pending
                self._rebuild_pending = False
                config = self._config
            if rebuild:
                self._rebuild(config)
                continue
            try:
                state = self._session.advance()
            except Exception as e:  # noqa: BLE001 - any solver failure ends or moves the drape, as the reference
                self._step_failed(str(e))
                continue
            now = time.monotonic()
            self._frame_times = [t for t in self._frame_times if now - t <= 1.0] + [now]
            self._publish()
            with self._cv:
                self._status.state = state
                self._status.fps = float(len(self._frame_times))
                self._status.simulated_seconds = self._session.time
                self._status.frames = self._session.result.frames_run
                if state == SS.STATE_FAILED:
                    self._status.message = self._session.result.message
                self._cv.notify_all()

    def _close_solver(self) -> None:
        s, self._solver = self._solver, None
        if s is not None and hasattr(s, "close"):
            s.close()

    def _rebuild(self, config: SimConfig) -> None:
        self._session = None
        self._close_solver()
        self._frame_times = []
        message, gpu_ok, backend = "", True, config.backend
        try:
            scene = config.scene()
            try:
                self._solver = self.factory(backend)
                self._solver.build(scene)  # device allocation can fail here too
            except Exception as e:  # noqa: BLE001
                if backend == CPU:
                    raise
                message = f"GPU unavailable: {e}; using CPU"
                self._gpu_note, gpu_ok, backend = message, False, CPU
                self._close_solver()
                self._solver = self.factory(backend)
                self._solver.build(scene)
            self._session = SS.DrapeSession(self._solver, list(config.garments), config.options)
        except Exception as e:  # noqa: BLE001
            self._session = None
            self._close_solver()
            with self._cv:
                self._status.state = SS.STATE_FAILED
                self._status.particles = 0
                self._status.fps = 0.0
                self._status.message = str(e)
                self._status.backend = backend
                self._cv.notify_all()
            return
        if not message and backend == CPU:
            message = self._gpu_note
        with self._cv:
            self._status.state = self._session.state
            self._status.particles = int(self._solver.particle_count())
            self._status.fps = 0.0
            self._status.simulated_seconds = 0.0
            self._status.frames = 0
            self._status.message = message
            self._status.backend = backend
            if not gpu_ok:
                self._status.gpu_available = False
            self._backend = backend
            self._revision += 1
            self._status.revision = self._revision
            self._cv.notify_all()
        self._publish()

    def _step_failed(self, what: str) -> None:
        if self._backend != CPU:
            self._gpu_note = f"GPU failed: {what}; using CPU"
            with self._cv:
                self._config = replace(self._config, backend=CPU)
                config = self._config
                self._status.gpu_available = False
            self._rebuild(config)
            return
        self._session = None
        self._frame_times = []
        with self._cv:
            self._status.state = SS.STATE_FAILED
            self._status.fps = 0.0
            self._status.message = what
            self._cv.notify_all()

    def _publish(self) -> None:
        self._frame += 1
        x = np.asarray(self._solver.positions(), np.float32)
        self.exchange.publish(PublishedFrame(self._revision, self._frame, x))
