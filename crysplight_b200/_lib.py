"""Loader for the in-tree sm_100a library ``crysplight_b200/lib/libcrysplight_cuda.so``.

There is no CPU fallback: if the library is missing or fails to load, every
entry point raises ``LibraryNotBuilt``.  Build it with ``crysplight_b200.build``
(or ``make -C crysplight_b200/csrc``).
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from .params import Box, Counters, OpticalParams, Readout, Records, TimeBinning

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.environ.get("CRYSPLIGHT_CUDA_LIB") or os.path.join(LIB_DIR, "libcrysplight_cuda.so")

# Exported symbols, exactly those declared in include/crysplight_cuda.h.
EXPORTS = (
    "cl_version", "cl_abi_version", "cl_create", "cl_destroy", "cl_last_error",
    "cl_run_photons", "cl_run_photons_device", "cl_run_segments",
    "cl_run_segments_device", "cl_sync", "cl_last_steps", "cl_set_launch",
    "cl_debug_eval", "cl_run_photons_noalloc", "cl_run_segments_moments_device",
    "cl_run_events_surrogate_device", "cl_surrogate_combine", "cl_debug_sampler",
    "cl_surrogate_inputs", "cl_set_time_budget", "cl_surrogate_combine_direct", "cl_surrogate_direct",
)

# Fixed-point scales of cl_run_segments_moments_device (crysplight_cuda.h)
MOMENT_T_SCALE = 1048576.0
MOMENT_T2_SCALE = 65536.0
MOMENT_T_MAX_NS = 4096.0

CL_OK = 0
CL_ERR_ARG = -1
CL_ERR_CUDA = -2
CL_ERR_OOM = -3
CL_ERR_TIMEOUT = -4
CL_ERR_STATE = -5

# include/crysplight_cuda.h: CL_MAX_BOUNCES_LIMIT, CL_DEFAULT_TIME_BUDGET_S
MAX_BOUNCES_LIMIT = 10_000_000
DEFAULT_TIME_BUDGET_S = 300.0


class LibraryNotBuilt(RuntimeError):
    pass


class CudaTransportError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


_lock = threading.Lock()
_lib = None

_P = C.c_void_p
_f = C.POINTER(C.c_float)


def _declare(lib: C.CDLL) -> None:
    lib.cl_version.restype = C.c_char_p
    lib.cl_abi_version.restype = C.c_int
    lib.cl_create.argtypes = [C.POINTER(C.c_void_p), C.c_int]
    lib.cl_create.restype = C.c_int
    lib.cl_destroy.argtypes = [_P]
    lib.cl_destroy.restype = None
    lib.cl_last_error.argtypes = [_P]
    lib.cl_last_error.restype = C.c_char_p
    common = [_P, C.POINTER(Box), C.POINTER(OpticalParams), C.POINTER(Readout),
              C.POINTER(TimeBinning)]
    lib.cl_run_photons.argtypes = common + [
        _P, _P, _P, _P, C.c_int32, C.c_int64, C.c_uint64, C.c_uint64, C.c_float, C.c_int32,
        _P, _P, C.POINTER(Counters), C.POINTER(Records)]
    lib.cl_run_photons.restype = C.c_int
    lib.cl_run_photons_device.argtypes = common + [
        _P, _P, _P, _P, C.c_int32, C.c_int64, C.c_uint64, C.c_uint64, C.c_float, C.c_int32,
        _P, _P, _P, C.POINTER(Records), _P]
    lib.cl_run_photons_device.restype = C.c_int
    lib.cl_run_segments.argtypes = common + [
        _P, _P, _P, _P, _P, _P, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, C.c_float,
        C.c_int32, _P, _P, _P, C.POINTER(Counters), C.POINTER(Records)]
    lib.cl_run_segments.restype = C.c_int
    lib.cl_run_segments_device.argtypes = common + [
        _P, _P, _P, _P, _P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, C.c_float,
        C.c_int32, _P, _P, _P, _P, C.POINTER(Records), _P]
    lib.cl_run_segments_device.restype = C.c_int
    lib.cl_run_segments_moments_device.argtypes = common + [
        _P, _P, _P, _P, _P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, C.c_float,
        C.c_int32, _P, _P, _P, _P, _P, _P, _P]
    lib.cl_run_segments_moments_device.restype = C.c_int
    lib.cl_sync.argtypes = [_P, _P]
    lib.cl_sync.restype = C.c_int
    lib.cl_last_steps.argtypes = [_P]
    lib.cl_last_steps.restype = C.c_int64
    lib.cl_set_launch.argtypes = [_P, C.c_int, C.c_int, C.c_int]
    lib.cl_set_launch.restype = C.c_int
    lib.cl_set_time_budget.argtypes = [_P, C.c_double]
    lib.cl_set_time_budget.restype = C.c_int
    lib.cl_debug_eval.argtypes = [_P, C.c_int, _P, _P, C.c_int64, C.c_uint64, C.c_int32]
    lib.cl_debug_eval.restype = C.c_int
    lib.cl_run_photons_noalloc.argtypes = common[1:] + [
        _P, _P, _P, _P, C.c_int32, C.c_int64, C.c_uint64, C.c_uint64, C.c_float, C.c_int32,
        _P, _P, C.POINTER(Counters), _P]
    lib.cl_run_photons_noalloc.restype = C.c_int
    lib.cl_run_events_surrogate_device.argtypes = common + [
        _P, _P, _P, _P, _P, _P, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, C.c_float, C.c_int32,
        _P, _P, _P, _P, _P, _P, _P, C.c_int64, C.c_uint64, C.c_int64, _P, _P, _P, _P, _P, _P]
    lib.cl_run_events_surrogate_device.restype = C.c_int
    lib.cl_surrogate_combine.argtypes = [_P, C.c_int32, C.c_int64, _P, _P, _P, C.POINTER(Box),
                                         C.POINTER(Readout), C.c_float, C.c_float, C.c_float,
                                         _P, _P, _P, _P, _P, _P]
    lib.cl_surrogate_combine.restype = C.c_int
    lib.cl_surrogate_combine_direct.argtypes = [_P, C.c_int32, C.c_int64, _P, _P, _P, _P, C.POINTER(Box),
                                                C.POINTER(Readout), C.c_float, C.c_float, C.c_float,
                                                _P, _P, _P, _P, _P, _P]
    lib.cl_surrogate_combine_direct.restype = C.c_int
    lib.cl_surrogate_direct.argtypes = [_P, C.c_int64, C.POINTER(Box), C.POINTER(OpticalParams),
                                        C.POINTER(Readout), _P, _P]
    lib.cl_surrogate_direct.restype = C.c_int
    lib.cl_surrogate_inputs.argtypes = [_P, C.c_int64, C.POINTER(Box), C.c_float, _P, _P]
    lib.cl_surrogate_inputs.restype = C.c_int
    lib.cl_debug_sampler.argtypes = [C.c_int, _P, C.c_int64, C.c_uint64, _P, _P, _P]
    lib.cl_debug_sampler.restype = C.c_int


def load() -> C.CDLL:
    """Load (once) and return the CUDA library; raise if it is not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise LibraryNotBuilt(
                    f"{LIB_PATH} not found: build the CUDA library first "
                    "(python -c 'import crysplight_b200.build as b; b.build()')")
            try:
                lib = C.CDLL(LIB_PATH)
            except OSError as e:
                raise LibraryNotBuilt(f"cannot load {LIB_PATH}: {e}") from e
            _declare(lib)
            _lib = lib
        return _lib


def check(lib: C.CDLL, handle, rc: int) -> None:
    if rc != CL_OK:
        msg = lib.cl_last_error(handle)
        raise CudaTransportError(rc, msg.decode() if msg else "unknown error")
