"""Learned light-response surrogate: an MLP from an emission point (x, y, z) to
the 64 per-SiPM detection probabilities and the 64 (mean, log sigma) pairs of
the detected photons' arrival times, trained on the GPU by the library's own
tcgen05 kernels (``csrc/cl_mlp.cu``: BF16 weights and activations, FP32
accumulation, Adam on FP32 master weights).

The reference has no surrogate; this is new in this framework.  The training
data is generated by the CUDA Monte Carlo itself (``scan_dataset``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib

D_IN, D_H, D_OUT = 3, 256, 192
N_CELLS = 64


def _declare(lib):
    if getattr(lib, "_mlp_declared", False):
        return
    P = C.c_void_p
    lib.cl_mlp_param_count.restype = C.c_int
    lib.cl_mlp_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int]
    lib.cl_mlp_create.restype = C.c_int
    lib.cl_mlp_destroy.argtypes = [P]
    lib.cl_mlp_destroy.restype = None
    lib.cl_mlp_last_error.argtypes = [P]
    lib.cl_mlp_last_error.restype = C.c_char_p
    lib.cl_mlp_set_params.argtypes = [P, P]
    lib.cl_mlp_get_params.argtypes = [P, P]
    lib.cl_mlp_set_data.argtypes = [P, P, P, C.c_int64]
    lib.cl_mlp_train.argtypes = [P, C.c_int, C.c_int, C.c_float, C.c_uint32, C.c_uint32,
                                 C.POINTER(C.c_float)]
    lib.cl_mlp_forward.argtypes = [P, P, P, C.c_int64]
    lib.cl_mlp_gradient.argtypes = [P, P, P, C.c_int, P, C.POINTER(C.c_float)]
    for n in ("cl_mlp_set_params", "cl_mlp_get_params", "cl_mlp_set_data", "cl_mlp_train",
              "cl_mlp_forward", "cl_mlp_gradient"):
        getattr(lib, n).restype = C.c_int
    lib._mlp_declared = True


def init_params(seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases (the usual
    linear-layer initialisation), in the cl_mlp parameter layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_out, fan_in in ((D_H, D_IN), (D_H, D_H), (D_H, D_H), (D_OUT, D_H)):
        b = 1.0 / np.sqrt(fan_in)
        parts.append(rng.uniform(-b, b, size=fan_out * fan_in))
        parts.append(rng.uniform(-b, b, size=fan_out))
    return np.concatenate(parts).astype(np.float32)


class MLP:
    """One network on one GPU (not re-entrant)."""

    def __init__(self, device: int = 0, max_batch: int = 65536, seed: int = 0):
        self.lib = _lib.load()
        _declare(self.lib)
        h = C.c_void_p()
        rc = self.lib.cl_mlp_create(C.byref(h), int(device), int(max_batch))
        if rc != 0:
            raise _lib.CudaTransportError(rc, "cl_mlp_create failed")
        self.h = h
        self.device = device
        self.max_batch = max_batch
        self.n_params = int(self.lib.cl_mlp_param_count())
        self.step = 0
        self.set_params(init_params(seed))

    def close(self):
        if getattr(self, "h", None):
            self.lib.cl_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise _lib.CudaTransportError(rc, self.lib.cl_mlp_last_error(self.h).decode())

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        self._check(self.lib.cl_mlp_set_params(self.h, C.c_void_p(p.ctypes.data)))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        self._check(self.lib.cl_mlp_get_params(self.h, C.c_void_p(p.ctypes.data)))
        return p

    def set_data(self, x, t):
        """x [n][3], t [n][192]: float32 CUDA tensors kept referenced here."""
        self._data = (x.contiguous(), t.contiguous())
        self._check(self.lib.cl_mlp_set_data(self.h, C.c_void_p(self._data[0].data_ptr()),
                                             C.c_void_p(self._data[1].data_ptr()), x.shape[0]))

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_float()
        self._check(self.lib.cl_mlp_train(self.h, int(steps), int(batch), float(lr), int(seed) & 0xFFFFFFFF,
                                          self.step & 0xFFFFFFFF, C.byref(loss)))
        self.step += steps
        return float(loss.value)

    def forward(self, x):
        import torch
        x = x.contiguous()
        out = torch.empty((x.shape[0], D_OUT), dtype=torch.float32, device=x.device)
        self._check(self.lib.cl_mlp_forward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                            x.shape[0]))
        return out

    def gradient(self, x, t):
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float()
        self._check(self.lib.cl_mlp_gradient(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                             x.shape[0], C.c_void_p(g.ctypes.data), C.byref(loss)))
        return float(loss.value), g
