"""ctypes binding of the learned preconditioner (include/drape_precond.h).

``LearnedPreconditioner`` owns a device network: parameters (FP32 master copy), training samples (Newton systems with
residual vectors), the forward pass (G and L = S G per slot), loss and gradient, z = L L^T r, and Adam training, all
on the GPU. ``init_params`` gives the initial parameters (He-normal hidden layers, zero output layer, so that the
initial preconditioner is block-Jacobi exactly). Nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import cuda as _cuda

_P = C.POINTER
_u8, _u32, _f, _d = C.c_uint8, C.c_uint32, C.c_float, C.c_double

HIDDEN, LAYERS = 64, 4
DEFECT, KAPORIN = 0, 1
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")


def _lib():
    L = _cuda.load()
    if getattr(L, "_precond_bound", False):
        return L
    L.drape_precond_param_count.restype = C.c_uint32
    L.drape_precond_param_count.argtypes = []
    L.drape_precond_create.argtypes = [C.c_int, _P(C.c_void_p)]
    L.drape_precond_destroy.argtypes = [C.c_void_p]
    L.drape_precond_destroy.restype = None
    L.drape_precond_last_error.argtypes = [C.c_void_p]
    L.drape_precond_last_error.restype = C.c_char_p
    L.drape_precond_set_params.argtypes = [C.c_void_p, _P(_f), C.c_size_t]
    L.drape_precond_get_params.argtypes = [C.c_void_p, _P(_f), C.c_size_t]
    L.drape_precond_add_sample.argtypes = [C.c_void_p, _u32, _P(_u32), _P(_u32), _P(_f), _P(_u8), _P(_u8), _P(_f),
                                           _u32, _P(C.c_int)]
    L.drape_precond_clear_samples.argtypes = [C.c_void_p]
    L.drape_precond_forward.argtypes = [C.c_void_p, C.c_int, _P(_f), _P(_f)]
    L.drape_precond_forward_inference.argtypes = [C.c_void_p, C.c_int, _P(_f)]
    L.drape_precond_loss_grad.argtypes = [C.c_void_p, C.c_int, C.c_int, _P(_d), _P(_f)]
    L.drape_precond_apply.argtypes = [C.c_void_p, C.c_int, _P(_f), _P(_f)]
    L.drape_precond_train.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_uint64, _P(_f)]
    L.drape_precond_set_objective.argtypes = [C.c_void_p, C.c_int]
    L.drape_precond_pcg.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _P(C.c_int), _P(_d)]
    L._precond_bound = True
    return L


def param_count() -> int:
    return int(_lib().drape_precond_param_count())


def param_shapes():
    """[(name, shape)] in the flat layout order of drape_precond_param_count()."""
    shapes = [("W_ne", (HIDDEN, 16)), ("b_ne", (HIDDEN,)), ("W_ee", (HIDDEN, 16)), ("b_ee", (HIDDEN,))]
    for l in range(LAYERS):
        shapes += [(f"W_m{l}", (HIDDEN, 2 * HIDDEN)), (f"b_m{l}", (HIDDEN,)),
                   (f"W_u{l}", (HIDDEN, 2 * HIDDEN)), (f"b_u{l}", (HIDDEN,))]
    return shapes + [("W_o", (16, 3 * HIDDEN)), ("b_o", (16,))]


def init_params(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = []
    for name, shape in param_shapes():
        if name.startswith("W_") and name != "W_o":
            out.append(rng.standard_normal(shape) * np.sqrt(2.0 / shape[1]))
        else:
            out.append(np.zeros(shape))
    return np.concatenate([a.reshape(-1) for a in out]).astype(np.float32)


def load_weights(name: str = "tube") -> np.ndarray:
    """Trained parameters shipped with the package (drape_b200/weights/<name>.npy)."""
    return np.load(os.path.join(WEIGHTS_DIR, f"{name}.npy")).astype(np.float32)


class LearnedPreconditioner:
    def __init__(self, device: int = 0, params: Optional[np.ndarray] = None):
        self.L = _lib()
        h = C.c_void_p()
        code = self.L.drape_precond_create(device, C.byref(h))
        _cuda._raise(code, self.L.drape_precond_last_error(None))
        self.h = h
        self.samples = []
        self.set_params(init_params(0) if params is None else params)

    def close(self):
        if self.h:
            self.L.drape_precond_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        _cuda._raise(code, self.L.drape_precond_last_error(self.h))

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        self._check(self.L.drape_precond_set_params(self.h, p.ctypes.data_as(_P(_f)), p.size))

    def params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        self._check(self.L.drape_precond_get_params(self.h, p.ctypes.data_as(_P(_f)), p.size))
        return p

    def add_sample(self, row_start, col_index, blocks, pinned, active, residuals) -> int:
        rs = np.ascontiguousarray(row_start, np.uint32)
        ci = np.ascontiguousarray(col_index, np.uint32)
        bl = np.ascontiguousarray(np.asarray(blocks).reshape(-1, 9), np.float32)
        pn = np.ascontiguousarray(pinned, np.uint8)
        ac = np.ascontiguousarray(active, np.uint8)
        res = np.ascontiguousarray(np.asarray(residuals, np.float32).reshape(-1, len(rs) - 1, 3))
        sid = C.c_int(-1)
        self._check(self.L.drape_precond_add_sample(self.h, len(rs) - 1, rs.ctypes.data_as(_P(_u32)),
                                                    ci.ctypes.data_as(_P(_u32)), bl.ctypes.data_as(_P(_f)),
                                                    pn.ctypes.data_as(_P(_u8)), ac.ctypes.data_as(_P(_u8)),
                                                    res.ctypes.data_as(_P(_f)), res.shape[0], C.byref(sid)))
        self.samples.append((len(rs) - 1, len(ci)))
        return sid.value

    def set_objective(self, objective: int) -> None:
        """KAPORIN (default; the samples' residual vectors are the random probes) or DEFECT."""
        self._check(self.L.drape_precond_set_objective(self.h, int(objective)))

    def clear_samples(self) -> None:
        self._check(self.L.drape_precond_clear_samples(self.h))
        self.samples = []

    def forward(self, sample: int):
        n, B = self.samples[sample]
        G = np.zeros((B, 3, 3), np.float32)
        Lb = np.zeros((B, 3, 3), np.float32)
        self._check(self.L.drape_precond_forward(self.h, sample, G.ctypes.data_as(_P(_f)), Lb.ctypes.data_as(_P(_f))))
        return G, Lb

    def forward_inference(self, sample: int) -> np.ndarray:
        """L per slot (B x 3 x 3) from the inference path the solver runs (drape_precond_forward_inference)."""
        n, B = self.samples[sample]
        Lb = np.zeros((B, 3, 3), np.float32)
        self._check(self.L.drape_precond_forward_inference(self.h, sample, Lb.ctypes.data_as(_P(_f))))
        return Lb

    def loss_grad(self, sample: int, residual: int = 0):
        loss = C.c_double()
        g = np.zeros(param_count(), np.float32)
        self._check(self.L.drape_precond_loss_grad(self.h, sample, residual, C.byref(loss), g.ctypes.data_as(_P(_f))))
        return loss.value, g

    def apply(self, sample: int, r) -> np.ndarray:
        n, _ = self.samples[sample]
        rr = np.ascontiguousarray(r, np.float32).reshape(n, 3)
        z = np.zeros((n, 3), np.float32)
        self._check(self.L.drape_precond_apply(self.h, sample, rr.ctypes.data_as(_P(_f)), z.ctypes.data_as(_P(_f))))
        return z

    def pcg(self, sample: int, rhs: int = 0, use_learned: bool = True, max_iterations: int = 500,
            tolerance: float = 1e-2):
        """(iterations, relative residual) of PCG on the sample's scaled system (drape_precond_pcg)."""
        it, rel = C.c_int(), C.c_double()
        self._check(self.L.drape_precond_pcg(self.h, sample, rhs, int(use_learned), max_iterations, tolerance,
                                             C.byref(it), C.byref(rel)))
        return it.value, rel.value

    def train(self, steps: int, lr: float = 1e-3, batch: int = 4, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(steps, 1), np.float32)
        self._check(self.L.drape_precond_train(self.h, steps, lr, batch, seed, losses.ctypes.data_as(_P(_f))))
        return losses[:steps]
