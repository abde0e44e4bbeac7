"""ctypes binding of libdrape_cuda.so (include/drape_cuda.h) with the reference's Solver interface on top.

``CudaSolver`` mirrors drape::sim::Solver (libs/sim/include/drape/sim/solver.hpp:85-98): build, update_fabric,
set_phase, step, read_positions (``positions()``), stats, snapshot, restore, range, particle_count; status codes map to
the reference's exception types (std::invalid_argument -> ValueError, std::out_of_range -> IndexError,
std::runtime_error "cuda: ..." -> CudaError). ``make_solver`` / ``is_available`` / ``backend_name`` mirror
makeSolver / isAvailable / backendName (libs/sim/src/solver_factory.cpp:16-61) for a "cuda" backend.

There is no CPU fallback here: if the library or a CUDA device is missing, creating a solver raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from . import build as _build
from .scene import (SceneDesc, drape_counters, drape_drape_options, drape_drape_result, drape_fabric,
                    drape_scene_desc, drape_stats)

_P = C.POINTER
_u8, _u32, _i32, _f, _d = C.c_uint8, C.c_uint32, C.c_int32, C.c_float, C.c_double

OK, INVALID, OUT_OF_RANGE, DEVICE_ERROR, NOT_BUILT = 0, -1, -2, -3, -4


class CudaError(RuntimeError):
    """std::runtime_error of the CUDA backend ("cuda: ...")."""


_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Loads libdrape_cuda.so (building it first when it is missing or stale and nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and (not os.path.exists(_build.LIB) or _build.stale()):
        _build.build()
    L = C.CDLL(_build.LIB)
    L.drape_cuda_version.restype = C.c_int
    L.drape_cuda_is_available.restype = C.c_int
    L.drape_cuda_create.argtypes = [C.c_int, _P(C.c_void_p)]
    L.drape_cuda_destroy.argtypes = [C.c_void_p]
    L.drape_cuda_destroy.restype = None
    L.drape_cuda_last_error.argtypes = [C.c_void_p]
    L.drape_cuda_last_error.restype = C.c_char_p
    L.drape_cuda_build.argtypes = [C.c_void_p, _P(drape_scene_desc)]
    L.drape_cuda_update_fabric.argtypes = [C.c_void_p, C.c_char_p, _P(drape_fabric), _u32]
    L.drape_cuda_set_phase.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
    L.drape_cuda_step.argtypes = [C.c_void_p, _d, C.c_int, C.c_int]
    L.drape_cuda_read_positions.argtypes = [C.c_void_p, _P(_f), C.c_size_t]
    L.drape_cuda_read_velocities.argtypes = [C.c_void_p, _P(_f), C.c_size_t]
    L.drape_cuda_stats.argtypes = [C.c_void_p, _P(drape_stats)]
    L.drape_cuda_snapshot_sizes.argtypes = [C.c_void_p, _P(_u32), _P(_u32), _P(_u32)]
    L.drape_cuda_snapshot.argtypes = [C.c_void_p, _P(_f), _P(_f), _P(_i32), _P(_d), _P(_f), _P(_d)]
    L.drape_cuda_restore.argtypes = [C.c_void_p, _P(_f), _P(_f), _u32, _P(_i32), _P(_d), _u32, _P(_f), _u32, _P(_d),
                                     _u32]
    L.drape_cuda_range.argtypes = [C.c_void_p, C.c_char_p, _P(_u32), _P(_u32)]
    L.drape_cuda_particle_count.argtypes = [C.c_void_p, _P(C.c_size_t)]
    L.drape_cuda_drape_to_rest.argtypes = [C.c_void_p, _P(C.c_char_p), _u32, _P(drape_drape_options),
                                           _P(drape_drape_result)]
    L.drape_cuda_counters.argtypes = [C.c_void_p, _P(drape_counters)]
    L.drape_cuda_reset_counters.argtypes = [C.c_void_p]
    L.drape_cuda_structure_sizes.argtypes = [C.c_void_p, _P(_u32)]
    L.drape_cuda_structure.argtypes = [C.c_void_p] + [_P(_u32)] * 9
    L.drape_cuda_contact_candidates.argtypes = [C.c_void_p, _P(_f), _P(_u8), _P(_f), _P(_f)]
    L.drape_cuda_capture_system.argtypes = [C.c_void_p, _d, _P(_f), _P(_f), _P(_u8)]
    L.drape_cuda_pcg.argtypes = [_u32, _P(_u32), _P(_u32), _P(_f), _P(_u8), _P(_u8), _P(_f), _P(_f), C.c_int, _d,
                                 _P(_f), _P(_f), _P(C.c_int)]
    L.drape_cuda_spmv_device.argtypes = [_u32, C.c_void_p, C.c_void_p, C.c_void_p, _u32, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
    L.drape_cuda_set_barrier_limit.argtypes = [C.c_void_p, C.c_uint64]
    L.drape_cuda_set_precond.argtypes = [C.c_void_p, C.c_void_p]
    L.drape_cuda_set_precond_schedule.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.drape_cuda_precond_factor.argtypes = [C.c_void_p, _P(_f)]
    L.drape_cuda_test_barrier_timeout.argtypes = [C.c_int, C.c_int, C.c_uint64, _P(C.c_int)]
    L.drape_cuda_inject_failure.argtypes = [C.c_void_p, C.c_int]
    L.drape_cuda_set_pcg_variant.argtypes = [C.c_void_p, C.c_int]
    L.drape_cuda_set_host_wait.argtypes = [C.c_void_p, C.c_uint32]
    L.drape_cuda_solve_threads.argtypes = [C.c_void_p, _P(C.c_int)]
    L.drape_cuda_runner_host_seconds.argtypes = [C.c_void_p, _P(_d)]
    L.drape_cuda_frame_times.argtypes = [C.c_void_p, _P(C.c_uint64), _P(C.c_uint64), C.c_size_t, _P(C.c_size_t)]
    L.drape_cuda_reduction_floor.argtypes = [C.c_int, C.c_int, C.c_int, _P(_d)]
    L.drape_cuda_cg_history.argtypes = [C.c_void_p, _P(_i32), C.c_size_t, _P(C.c_size_t)]
    L.drape_cuda_stream.argtypes = [C.c_void_p, _P(C.c_void_p)]
    L.drape_cuda_profile.argtypes = [C.c_void_p, C.c_int]
    L.drape_cuda_profile_read.argtypes = [C.c_void_p, _P(drape_profile)]
    L.drape_cuda_transfer_bytes.argtypes = [C.c_void_p, _P(C.c_uint64), _P(C.c_uint64)]
    L.drape_cuda_pcg_noalloc.argtypes = [_u32, _u32, C.c_void_p, C.c_void_p, C.c_void_p, _u32, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, _d, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
    _lib = L
    return L


KERNEL_NAMES = ("k_begin", "k_activate", "k_assemble", "k_solve", "k_finish", "k_stats", "net_forward")


class drape_profile(C.Structure):
    _fields_ = [("launches", C.c_int64 * 7), ("milliseconds", C.c_double * 7), ("cg_iterations", C.c_int64),
                ("energy_evaluations", C.c_int64)]


def _raise(code: int, msg) -> None:
    if code == OK:
        return
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    if code == INVALID:
        raise ValueError(msg)
    if code == OUT_OF_RANGE:
        raise IndexError(msg)
    raise CudaError(msg)


def _np(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a, ctype):
    return a.ctypes.data_as(_P(ctype))


def backend_name() -> str:
    return "cuda"


def is_available() -> bool:
    try:
        return bool(load().drape_cuda_is_available())
    except OSError:
        return False


class CudaSolver:
    """The reference's Solver interface on one B200."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        code = self.L.drape_cuda_create(device, C.byref(h))
        _raise(code, self.L.drape_cuda_last_error(None))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.drape_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        _raise(code, self.L.drape_cuda_last_error(self.h))

    # ---- Solver ----
    def build(self, scene) -> None:
        self._desc = SceneDesc(scene)
        self._check(self.L.drape_cuda_build(self.h, self._desc.ptr()))

    def update_fabric(self, garment: str, fabrics) -> None:
        arr = (drape_fabric * max(1, len(fabrics)))(*[f.to_c() for f in fabrics])
        self._check(self.L.drape_cuda_update_fabric(self.h, garment.encode(), arr, len(fabrics)))

    def set_phase(self, garment: str, phase: int) -> None:
        self._check(self.L.drape_cuda_set_phase(self.h, garment.encode(), int(phase)))

    def step(self, dt: float = 1.0 / 60.0, substeps: int = 2, iterations: int = 2) -> None:
        self._check(self.L.drape_cuda_step(self.h, dt, substeps, iterations))

    def particle_count(self) -> int:
        n = C.c_size_t()
        self._check(self.L.drape_cuda_particle_count(self.h, C.byref(n)))
        return n.value

    def positions(self) -> np.ndarray:
        n = self.particle_count()
        out = np.zeros((n, 3), np.float32)
        self._check(self.L.drape_cuda_read_positions(self.h, _p(out, _f), n))
        return out

    def read_positions(self, out: np.ndarray) -> None:
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.ndim != 2 or out.shape[1] != 3:
            raise ValueError("readPositions: out must be a contiguous (n, 3) float32 array")
        self._check(self.L.drape_cuda_read_positions(self.h, _p(out, _f), out.shape[0]))

    def velocities(self) -> np.ndarray:
        n = self.particle_count()
        out = np.zeros((n, 3), np.float32)
        self._check(self.L.drape_cuda_read_velocities(self.h, _p(out, _f), n))
        return out

    def stats(self) -> drape_stats:
        st = drape_stats()
        self._check(self.L.drape_cuda_stats(self.h, C.byref(st)))
        return st

    def snapshot(self) -> dict:
        n, g, k = _u32(), _u32(), _u32()
        self._check(self.L.drape_cuda_snapshot_sizes(self.h, C.byref(n), C.byref(g), C.byref(k)))
        n, g, k = n.value, g.value, k.value
        snap = dict(positions=np.zeros((n, 3), np.float32), velocities=np.zeros((n, 3), np.float32),
                    phases=np.zeros(g, np.int32), assembly_time=np.zeros(g), seam_start_gap=np.zeros(k, np.float32),
                    contact_force=np.zeros(n))
        self._check(self.L.drape_cuda_snapshot(self.h, _p(snap["positions"], _f), _p(snap["velocities"], _f),
                                               _p(snap["phases"], _i32), _p(snap["assembly_time"], _d),
                                               _p(snap["seam_start_gap"], _f), _p(snap["contact_force"], _d)))
        return snap

    def restore(self, snap: dict) -> None:
        pos, vel = _np(snap["positions"], np.float32), _np(snap["velocities"], np.float32)
        ph, at = _np(snap["phases"], np.int32), _np(snap["assembly_time"], np.float64)
        sg, cf = _np(snap["seam_start_gap"], np.float32), _np(snap["contact_force"], np.float64)
        self._check(self.L.drape_cuda_restore(self.h, _p(pos, _f), _p(vel, _f), len(pos), _p(ph, _i32), _p(at, _d),
                                              len(ph), _p(sg, _f), len(sg), _p(cf, _d), len(cf)))

    def range(self, garment: str):
        off, cnt = _u32(), _u32()
        self._check(self.L.drape_cuda_range(self.h, garment.encode(), C.byref(off), C.byref(cnt)))
        return off.value, cnt.value

    # ---- beyond the Solver interface ----
    def drape_to_rest(self, garments: Sequence[str], options: Optional[drape_drape_options] = None):
        ids = (C.c_char_p * len(garments))(*[g.encode() for g in garments])
        res = drape_drape_result()
        opt = C.byref(options) if options is not None else None
        self._check(self.L.drape_cuda_drape_to_rest(self.h, ids, len(garments), opt, C.byref(res)))
        return res

    def counters(self) -> drape_counters:
        c = drape_counters()
        self._check(self.L.drape_cuda_counters(self.h, C.byref(c)))
        return c

    def reset_counters(self) -> None:
        self._check(self.L.drape_cuda_reset_counters(self.h))

    def structure(self) -> dict:
        sz = (_u32 * 5)()
        self._check(self.L.drape_cuda_structure_sizes(self.h, sz))
        n, B, S, H, K = list(sz)
        out = dict(row_start=np.zeros(n + 1, np.uint32), col_index=np.zeros(B, np.uint32),
                   diag_slot=np.zeros(n, np.uint32), stretch_slots=np.zeros((S, 9), np.uint32),
                   hinge_slots=np.zeros((H, 16), np.uint32), seam_slots=np.zeros((K, 4), np.uint32),
                   stretch_v=np.zeros((S, 3), np.uint32), hinge_v=np.zeros((H, 4), np.uint32),
                   seam_ab=np.zeros((K, 2), np.uint32))
        keys = ["row_start", "col_index", "diag_slot", "stretch_slots", "hinge_slots", "seam_slots", "stretch_v",
                "hinge_v", "seam_ab"]
        self._check(self.L.drape_cuda_structure(self.h, *[_p(out[k], _u32) for k in keys]))
        return out

    def contact_candidates(self, x_start: np.ndarray):
        xs = _np(x_start, np.float32)
        n = len(xs)
        near, nrm, off = np.zeros(n, np.uint8), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        self._check(self.L.drape_cuda_contact_candidates(self.h, _p(xs, _f), _p(near, _u8), _p(nrm, _f), _p(off, _f)))
        return near, nrm, off

    def capture_system(self, h: float) -> dict:
        st = self.structure()
        n, B = len(st["diag_slot"]), len(st["col_index"])
        blocks, grad, active = np.zeros((B, 3, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.uint8)
        self._check(self.L.drape_cuda_capture_system(self.h, h, _p(blocks, _f), _p(grad, _f), _p(active, _u8)))
        return dict(blocks=blocks, grad=grad, active=active, **st)

    def cg_history(self, capacity: int = 1 << 16) -> np.ndarray:
        out = np.zeros(capacity, np.int32)
        cnt = C.c_size_t()
        self._check(self.L.drape_cuda_cg_history(self.h, _p(out, _i32), capacity, C.byref(cnt)))
        return out[:cnt.value]

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._check(self.L.drape_cuda_stream(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, enable, solve_only: bool = False) -> None:
        """Per-kernel CUDA-event timing on the solver's stream: every kernel, or (solve_only) k_solve alone, which
        adds two events a Newton iteration instead of two around every launch."""
        self._check(self.L.drape_cuda_profile(self.h, (2 if solve_only else 1) if enable else 0))

    def profile_read(self) -> dict:
        p = drape_profile()
        self._check(self.L.drape_cuda_profile_read(self.h, C.byref(p)))
        return dict(launches={k: int(p.launches[i]) for i, k in enumerate(KERNEL_NAMES)},
                    milliseconds={k: float(p.milliseconds[i]) for i, k in enumerate(KERNEL_NAMES)},
                    cg_iterations=int(p.cg_iterations), energy_evaluations=int(p.energy_evaluations))

    def transfer_bytes(self):
        a, b = C.c_uint64(), C.c_uint64()
        self._check(self.L.drape_cuda_transfer_bytes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_barrier_limit(self, nanoseconds: int) -> None:
        self._check(self.L.drape_cuda_set_barrier_limit(self.h, int(nanoseconds)))

    def set_precond(self, precond) -> None:
        """Use a LearnedPreconditioner's current parameters for the Newton solves (None: block-Jacobi)."""
        self._check(self.L.drape_cuda_set_precond(self.h, None if precond is None else precond.h))

    def precond_factor(self) -> np.ndarray:
        """L per slot (B, 3, 3) from the solver's last network run."""
        B = len(self.structure()["col_index"])
        out = np.zeros((B, 3, 3), np.float32)
        self._check(self.L.drape_cuda_precond_factor(self.h, _p(out, _f)))
        return out

    def set_precond_schedule(self, refresh_every: int = 1, jacobi_first: int = 0) -> None:
        self._check(self.L.drape_cuda_set_precond_schedule(self.h, int(refresh_every), int(jacobi_first)))

    def runner_host_seconds(self):
        """Host seconds of the last drape_to_rest: (set-up, frame loop, rest of the call)."""
        out = (_d * 3)()
        self._check(self.L.drape_cuda_runner_host_seconds(self.h, out))
        return tuple(out)

    def frame_times(self, capacity: int = 1 << 16):
        """(begin, end) device timestamps in ns of the frames run in batches since the last call, as an (n, 2) array."""
        b = np.zeros(capacity, np.uint64)
        e = np.zeros(capacity, np.uint64)
        n = C.c_size_t()
        self._check(self.L.drape_cuda_frame_times(self.h, b.ctypes.data_as(_P(C.c_uint64)),
                                                  e.ctypes.data_as(_P(C.c_uint64)), capacity, C.byref(n)))
        return np.stack([b[:n.value], e[:n.value]], axis=1)

    def set_host_wait(self, spin_microseconds: int) -> None:
        """Host wait: poll for up to spin_microseconds, then sleep between polls (2**32 - 1: poll only)."""
        self._check(self.L.drape_cuda_set_host_wait(self.h, int(spin_microseconds)))

    def set_pcg_variant(self, variant: int) -> None:
        """0: the reference-order block-Jacobi PCG (default; resident rows where the scene fits); 1: pipelined, one
        grid exchange per iteration; 2: Chronopoulos-Gear, one reduction and one plain barrier per iteration; 3: the
        reference order on the 1024-thread kernel (bit-identical to 0)."""
        self._check(self.L.drape_cuda_set_pcg_variant(self.h, int(variant)))

    def solve_threads(self) -> int:
        """Threads per block of the built scene's solve kernel: 512 (resident rows) or 1024."""
        t = C.c_int(0)
        self._check(self.L.drape_cuda_solve_threads(self.h, C.byref(t)))
        return t.value

    def inject_failure(self, steps: int) -> None:
        self._check(self.L.drape_cuda_inject_failure(self.h, int(steps)))


def make_solver(backend: str = "cuda", device: int = 0) -> CudaSolver:
    """makeSolver for the "cuda" backend: raises CudaError naming the backend when it is unavailable."""
    if backend != "cuda":
        raise ValueError(f"unknown solver backend '{backend}'")
    return CudaSolver(device)


def pcg(row_start, col_index, blocks, pinned, active, normals, grad, max_iterations=50, tolerance=1e-2):
    """The device PCG on a host-given system (see drape_cuda_pcg)."""
    L = load()
    n = len(row_start) - 1
    rs, ci = _np(row_start, np.uint32), _np(col_index, np.uint32)
    bl = _np(blocks, np.float32).reshape(-1, 9)
    pn, ac = _np(pinned, np.uint8), _np(active, np.uint8)
    nm, g = _np(normals, np.float32), _np(grad, np.float32)
    step, resid, its = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), C.c_int()
    code = L.drape_cuda_pcg(n, _p(rs, _u32), _p(ci, _u32), _p(bl, _f), _p(pn, _u8), _p(ac, _u8), _p(nm, _f), _p(g, _f),
                            max_iterations, tolerance, _p(step, _f), _p(resid, _f), C.byref(its))
    _raise(code, L.drape_cuda_last_error(None))
    return step, resid, its.value


def test_barrier_timeout(device: int = 0, blocks: int = 2, nanoseconds: int = 20_000_000) -> int:
    L = load()
    st = C.c_int(-1)
    _raise(L.drape_cuda_test_barrier_timeout(device, blocks, nanoseconds, C.byref(st)), L.drape_cuda_last_error(None))
    return st.value


def reduction_floor(device: int = 0, mode: int = 0, iterations: int = 2000) -> float:
    """Device microseconds per round of the persistent solve's grid-wide exchanges with no other work
    (drape_cuda_reduction_floor): mode 0 = the two FP64 reductions of a reference-order PCG iteration, 1 = one merged
    reduction plus a plain barrier, 2 = one merged reduction, 3 = two plain barriers; 4-7 = modes 0-3 on the
    resident-row solve's grid (one 512-thread block per SM)."""
    L = load()
    ns = C.c_double(0.0)
    _raise(L.drape_cuda_reduction_floor(device, mode, iterations, C.byref(ns)), L.drape_cuda_last_error(None))
    return ns.value / 1000.0
