"""ctypes binding of the collision-field bake (include/drape_bake.h): bakeCollisionField
(libs/avatar/src/collision_bake.cpp:98-208) on a B200. ``bake_field`` returns a scene.Field ready for a Scene's body.
There is no CPU fallback: without a usable device the call raises CudaError.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence, Tuple

import numpy as np

from . import cuda as _cuda
from .meshes import TriangleMesh
from .scene import Field

_P = C.POINTER


class drape_mesh_desc(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("vertices", _P(C.c_double)), ("triangle_count", C.c_uint32),
                ("triangles", _P(C.c_uint32))]


class drape_bake_options(C.Structure):
    _fields_ = [("cell_size", C.c_double), ("padding", C.c_double), ("band", C.c_double)]


def _lib():
    L = _cuda.load()
    if getattr(L, "_bake_bound", False):
        return L
    L.drape_bake_grid.argtypes = [_P(drape_mesh_desc), C.c_uint32, _P(drape_bake_options), _P(C.c_double),
                                  _P(C.c_int32)]
    L.drape_bake_field.argtypes = [C.c_int, _P(drape_mesh_desc), C.c_uint32, _P(drape_bake_options),
                                   _P(C.c_float), C.c_size_t]
    L.drape_bake_last_ms.restype = C.c_double
    L.drape_bake_last_error.restype = C.c_char_p
    L._bake_bound = True
    return L


class MeshArray:
    """Contiguous copies of the components and the drape_mesh_desc array that points at them."""

    def __init__(self, components: Sequence[TriangleMesh]):
        self._keep = []
        self.descs = (drape_mesh_desc * max(1, len(components)))()
        for k, m in enumerate(components):
            v = np.ascontiguousarray(m.vertices, np.float64).reshape(-1)
            t = np.ascontiguousarray(m.triangles, np.uint32).reshape(-1)
            self._keep += [v, t]
            self.descs[k] = drape_mesh_desc(len(v) // 3, v.ctypes.data_as(_P(C.c_double)), len(t) // 3,
                                            t.ctypes.data_as(_P(C.c_uint32)))
        self.count = len(components)


def options(cell_size: float = 0.004, padding: float = 0.05, band: float = 0.02) -> drape_bake_options:
    """BakeOptions (collision_bake.hpp:10-14)."""
    return drape_bake_options(cell_size, padding, band)


def bake_grid(components: Sequence[TriangleMesh], opts: drape_bake_options = None) -> Tuple[np.ndarray, tuple]:
    L = _lib()
    opts = opts or options()
    arr = MeshArray(components)
    origin, dims = (C.c_double * 3)(), (C.c_int32 * 3)()
    _cuda._raise(L.drape_bake_grid(arr.descs, arr.count, C.byref(opts), origin, dims), L.drape_bake_last_error())
    return np.array(origin[:]), tuple(int(d) for d in dims)


def bake_field(components: Sequence[TriangleMesh], opts: drape_bake_options = None, device: int = 0) -> Field:
    """The collision field of the union of the closed components, baked on the GPU."""
    L = _lib()
    opts = opts or options()
    origin, dims = bake_grid(components, opts)
    arr = MeshArray(components)
    values = np.zeros(dims[0] * dims[1] * dims[2], np.float32)
    _cuda._raise(L.drape_bake_field(device, arr.descs, arr.count, C.byref(opts), values.ctypes.data_as(_P(C.c_float)),
                                    values.size), L.drape_bake_last_error())
    return Field(origin, float(opts.cell_size), dims, float(opts.band), values.reshape(dims[2], dims[1], dims[0]))


def last_ms() -> float:
    """Device time of this thread's last bake (drape_bake_last_ms)."""
    return float(_lib().drape_bake_last_ms())
