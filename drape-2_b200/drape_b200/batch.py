"""ctypes binding of the batched drapes (include/drape_batch.h).

``BatchSolver`` advances many independent garments, each on its own body, on one GPU: one persistent solve launch
per Newton iteration for all of them (each garment with its own PCG, line search and convergence test), frames
replayed from a CUDA graph, and an autotuned solve variant. ``shard`` splits a list of garments across ranks for
multi-GPU batches (no collective on the data path: every rank drapes its own garments).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import cuda as _cuda
from .scene import (SceneDesc, drape_counters, drape_drape_options, drape_drape_result, drape_scene_desc,
                    drape_stats)

_P = C.POINTER
_u32, _u64, _f, _d = C.c_uint32, C.c_uint64, C.c_float, C.c_double


class drape_batch_tuning(C.Structure):
    _fields_ = [("row_lanes", C.c_int32), ("block_threads", C.c_int32), ("blocks", C.c_int32),
                ("variants_timed", C.c_int32), ("ms_per_newton", C.c_double)]


class drape_batch_profile(C.Structure):
    _fields_ = [("frames", C.c_int64), ("graph_launches", C.c_int64), ("solve_launches", C.c_int64),
                ("solve_ms", C.c_double), ("frame_ms", C.c_double), ("kernel_launches", C.c_int64),
                ("cg_iterations", C.c_int64), ("pcg_bytes", C.c_double)]


def _lib():
    L = _cuda.load()
    if getattr(L, "_batch_bound", False):
        return L
    vp = C.c_void_p
    L.drape_batch_create.argtypes = [C.c_int, _P(vp)]
    L.drape_batch_destroy.argtypes = [vp]
    L.drape_batch_destroy.restype = None
    L.drape_batch_last_error.argtypes = [vp]
    L.drape_batch_last_error.restype = C.c_char_p
    L.drape_batch_add.argtypes = [vp, _P(drape_scene_desc), _P(_u32)]
    L.drape_batch_build.argtypes = [vp]
    L.drape_batch_set_precond.argtypes = [vp, vp]
    L.drape_batch_autotune.argtypes = [vp, C.c_int, _P(drape_batch_tuning)]
    L.drape_batch_set_tuning.argtypes = [vp, _P(drape_batch_tuning)]
    L.drape_batch_step.argtypes = [vp, _d, C.c_int, C.c_int]
    L.drape_batch_set_phase.argtypes = [vp, _u32, C.c_int]
    L.drape_batch_drape_to_rest.argtypes = [vp, _P(drape_drape_options), _P(drape_drape_result), _P(_d), _u32]
    L.drape_batch_size.argtypes = [vp, _P(_u32), _P(_u64), _P(_u64)]
    L.drape_batch_particle_count.argtypes = [vp, _u32, _P(_u32)]
    L.drape_batch_read_positions.argtypes = [vp, _u32, _P(_f), C.c_size_t]
    L.drape_batch_stats.argtypes = [vp, _u32, _P(drape_stats)]
    L.drape_batch_counters.argtypes = [vp, _u32, _P(drape_counters)]
    L.drape_batch_reset_counters.argtypes = [vp]
    L.drape_batch_save.argtypes = [vp]
    L.drape_batch_restore.argtypes = [vp]
    L.drape_batch_set_profiling.argtypes = [vp, C.c_int]
    L.drape_batch_profile_read.argtypes = [vp, _P(drape_batch_profile)]
    L.drape_batch_stream.argtypes = [vp, _P(vp)]
    L._batch_bound = True
    return L


def shard(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Garment indices per rank: largest first onto the least-loaded rank (load = particle count), so every rank
    drapes about the same work. Deterministic; ranks are independent afterwards."""
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for g in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(g)
        load[r] += int(sizes[g])
    return [sorted(x) for x in out]


class BatchSolver:
    def __init__(self, device: int = 0):
        self.L = _lib()
        h = C.c_void_p()
        _cuda._raise(self.L.drape_batch_create(device, C.byref(h)), self.L.drape_batch_last_error(None))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.drape_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        _cuda._raise(code, self.L.drape_batch_last_error(self.h))

    def add(self, scene) -> int:
        desc = SceneDesc(scene)
        idx = _u32()
        self._check(self.L.drape_batch_add(self.h, desc.ptr(), C.byref(idx)))
        return idx.value

    def build(self) -> None:
        self._check(self.L.drape_batch_build(self.h))

    def set_precond(self, precond) -> None:
        self._check(self.L.drape_batch_set_precond(self.h, None if precond is None else precond.h))

    def autotune(self, frames: int = 2) -> dict:
        t = drape_batch_tuning()
        self._check(self.L.drape_batch_autotune(self.h, frames, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def set_tuning(self, row_lanes: int, block_threads: int) -> dict:
        t = drape_batch_tuning(row_lanes, block_threads, 0, 0, 0.0)
        self._check(self.L.drape_batch_set_tuning(self.h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def step(self, dt: float = 1.0 / 60.0, substeps: int = 1, iterations: int = 2) -> None:
        self._check(self.L.drape_batch_step(self.h, dt, substeps, iterations))

    def set_phase(self, index: int, phase: int) -> None:
        self._check(self.L.drape_batch_set_phase(self.h, index, int(phase)))

    def drape_to_rest(self, options: Optional[drape_drape_options] = None):
        """Drapes every garment to rest; returns (results, settle_seconds) per garment."""
        g = self.size()[0]
        res = (drape_drape_result * g)()
        secs = np.zeros(g, np.float64)
        opt = C.byref(options) if options is not None else None
        self._check(self.L.drape_batch_drape_to_rest(self.h, opt, res, secs.ctypes.data_as(_P(_d)), g))
        return list(res), secs

    def size(self):
        g, n, b = _u32(), _u64(), _u64()
        self._check(self.L.drape_batch_size(self.h, C.byref(g), C.byref(n), C.byref(b)))
        return g.value, n.value, b.value

    def particle_count(self, index: int) -> int:
        n = _u32()
        self._check(self.L.drape_batch_particle_count(self.h, index, C.byref(n)))
        return n.value

    def positions(self, index: int) -> np.ndarray:
        n = self.particle_count(index)
        out = np.zeros((n, 3), np.float32)
        self._check(self.L.drape_batch_read_positions(self.h, index, out.ctypes.data_as(_P(_f)), n))
        return out

    def stats(self, index: int) -> drape_stats:
        st = drape_stats()
        self._check(self.L.drape_batch_stats(self.h, index, C.byref(st)))
        return st

    def counters(self, index: int) -> drape_counters:
        c = drape_counters()
        self._check(self.L.drape_batch_counters(self.h, index, C.byref(c)))
        return c

    def reset_counters(self) -> None:
        self._check(self.L.drape_batch_reset_counters(self.h))

    def save(self) -> None:
        self._check(self.L.drape_batch_save(self.h))

    def restore(self) -> None:
        self._check(self.L.drape_batch_restore(self.h))

    def profile(self, enable: bool) -> None:
        self._check(self.L.drape_batch_set_profiling(self.h, 1 if enable else 0))

    def profile_read(self) -> dict:
        p = drape_batch_profile()
        self._check(self.L.drape_batch_profile_read(self.h, C.byref(p)))
        return {k: getattr(p, k) for k, _ in p._fields_}

    def stream_handle(self) -> int:
        p = C.c_void_p()
        self._check(self.L.drape_batch_stream(self.h, C.byref(p)))
        return p.value or 0
