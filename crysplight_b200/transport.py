"""Host-side mirror of CryspLight's transport call, backed by the sm_100a library.

``run_photons_ka`` has the keyword signature of the reference's
``run_photons_ka!`` (src/kernel.jl:312-319) and returns the same
``Accumulator`` (plus per-photon records with ``return_records=True``);
``run_photons`` has the signature of the CPU reference ``run_photons!``
(src/transport.jl:245-249).  Both run on the GPU through the C-ABI; there is
no CPU fallback.  ``run_segments`` is the batched per-point / per-event form
(the event pipeline's flush!, src/events.jl:65-91, without the batch limit).
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .params import (Accumulator, Box, Counters, OpticalParams, PhotonRecords, Readout,
                     Records, SipmGrid, TimeBinning, COUNTER_NAMES)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else C.c_void_p(a.ctypes.data)


# cudaStreamLegacy: the legacy default stream, named explicitly because the
# C-ABI reads a NULL stream as the handle's own stream.
CUDA_STREAM_LEGACY = 1


def stream_arg(stream):
    """The C-ABI stream argument for a CUDA stream handle: None -> NULL (the
    library handle's stream); 0, torch's default stream -> cudaStreamLegacy,
    so that the call is ordered with the default stream's work."""
    if stream is None:
        return None
    return C.c_void_p(int(stream) or CUDA_STREAM_LEGACY)


def _as_readout(ro) -> Readout:
    return ro if isinstance(ro, Readout) else Readout(ro)


def _positions(pos, positions) -> np.ndarray:
    if positions is None:
        if pos is None:
            raise ValueError("pass pos or positions")
        positions = [pos]
    p = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    if p.shape[0] < 1:
        raise ValueError("positions must not be empty")
    return np.ascontiguousarray(p)


@dataclass
class SegmentResult:
    """Per-segment outputs of ``run_segments``."""
    maps: np.ndarray        # (nx, ny, n_segments) uint32, Fortran order
    tmin: np.ndarray        # (nx, ny, n_segments) float32, +Inf where no detection
    npe: np.ndarray         # (n_segments,) int32
    counters: dict


class Engine:
    """One library handle bound to a CUDA device (not re-entrant)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.cl_create(C.byref(h), int(device))
        if rc != _lib.CL_OK:
            msg = self.lib.cl_last_error(None)
            raise _lib.CudaTransportError(rc, msg.decode() if msg else "cl_create failed")
        self.handle = h
        self.device = device
        self._lock = threading.Lock()

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.cl_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        _lib.check(self.lib, self.handle, rc)

    @property
    def last_steps(self) -> int:
        """Bounce-loop iterations executed by the last completed call."""
        return int(self.lib.cl_last_steps(self.handle))

    def set_launch(self, ctas_per_sm: int = 0, threads_per_cta: int = 0, warp_chunk: int = 0) -> None:
        self._check(self.lib.cl_set_launch(self.handle, ctas_per_sm, threads_per_cta, warp_chunk))

    def set_time_budget(self, seconds: float) -> None:
        """Device time budget of every transport launch on this engine (0 = none):
        a launch that runs longer stops and the call raises CL_ERR_TIMEOUT."""
        self._check(self.lib.cl_set_time_budget(self.handle, float(seconds)))

    # -- run_photons_ka!, src/kernel.jl:312-367 --------------------------------
    def run_photons_ka(self, box: Box, op: OpticalParams, ro, tb: TimeBinning, *,
                       n_photons: int, seed: int, pos=None, positions=None, t0s=None,
                       pid_offset: int = 0, tau_ns: float, max_bounces: int = 100_000,
                       return_records: bool = False):
        ro = _as_readout(ro)
        p = _positions(pos, positions)
        npos = p.shape[0]
        px, py, pz = (np.ascontiguousarray(p[:, i]) for i in range(3))
        pt = None
        if t0s is not None:
            pt = np.ascontiguousarray(np.asarray(t0s, dtype=np.float32).reshape(-1))
            if pt.shape[0] != npos:
                raise ValueError("t0s must have one entry per position")
        if int(n_photons) < 0:
            raise ValueError("n_photons must be >= 0")
        if int(seed) < 0 or int(pid_offset) < 0:
            raise ValueError("seed and pid_offset must be non-negative (UInt64 in the reference)")
        acc = Accumulator.empty(ro.grid, tb)
        ctr = Counters()
        recs = PhotonRecords.empty(int(n_photons)) if return_records else None
        crec = recs.as_c() if recs is not None else None
        with self._lock:
            rc = self.lib.cl_run_photons(
                self.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
                _ptr(px), _ptr(py), _ptr(pz), _ptr(pt), npos, int(n_photons),
                int(seed) & 0xFFFFFFFFFFFFFFFF, int(pid_offset), float(np.float32(tau_ns)),
                int(max_bounces), _ptr(acc.counts), _ptr(acc.first_ns), C.byref(ctr),
                C.byref(crec) if crec is not None else None)
            self._check(rc)
        acc.set_counters(ctr)
        return (acc, recs) if return_records else acc

    # -- run_photons!, src/transport.jl:245-273 --------------------------------
    def run_photons(self, box: Box, op: OpticalParams, ro, tb: TimeBinning, *,
                    n_photons: int, seed: int, pos=None, positions=None, tau_ns: float,
                    max_bounces: int = 100_000) -> Accumulator:
        return self.run_photons_ka(box, op, ro, tb, n_photons=n_photons, seed=seed, pos=pos,
                                   positions=positions, tau_ns=tau_ns, max_bounces=max_bounces)

    # -- batched segments (scan points / events) -------------------------------
    def run_segments(self, box: Box, op: OpticalParams, ro, tb: TimeBinning, *,
                     sources: np.ndarray, photons_per_source: Sequence[int],
                     segment_of_source: Sequence[int], n_segments: int, seed: int,
                     t0s=None, pid_offset: int = 0, tau_ns: float,
                     max_bounces: int = 100_000, return_records: bool = False):
        ro = _as_readout(ro)
        s = np.ascontiguousarray(np.asarray(sources, dtype=np.float32).reshape(-1, 3))
        n_src = s.shape[0]
        cnt = np.asarray(photons_per_source, dtype=np.int64).reshape(-1)
        seg = np.ascontiguousarray(np.asarray(segment_of_source, dtype=np.int32).reshape(-1))
        if cnt.shape[0] != n_src or seg.shape[0] != n_src:
            raise ValueError("one photon count and one segment id per source")
        if (cnt < 0).any():
            raise ValueError("photon counts must be >= 0")
        off = np.zeros(n_src + 1, np.int64)
        np.cumsum(cnt, out=off[1:])
        sx, sy, sz = (np.ascontiguousarray(s[:, i]) for i in range(3))
        st = None
        if t0s is not None:
            st = np.ascontiguousarray(np.asarray(t0s, dtype=np.float32).reshape(-1))
            if st.shape[0] != n_src:
                raise ValueError("t0s must have one entry per source")
        nx, ny = ro.grid.nx, ro.grid.ny
        maps = np.zeros((nx, ny, int(n_segments)), np.uint32, order="F")
        tmin = np.zeros((nx, ny, int(n_segments)), np.float32, order="F")
        npe = np.zeros(int(n_segments), np.int32)
        ctr = Counters()
        n = int(off[-1])
        recs = PhotonRecords.empty(n) if return_records else None
        crec = recs.as_c() if recs is not None else None
        with self._lock:
            rc = self.lib.cl_run_segments(
                self.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
                _ptr(sx), _ptr(sy), _ptr(sz), _ptr(st), _ptr(off), _ptr(seg), n_src,
                int(n_segments), int(seed) & 0xFFFFFFFFFFFFFFFF, int(pid_offset),
                float(np.float32(tau_ns)), int(max_bounces), _ptr(maps), _ptr(tmin), _ptr(npe),
                C.byref(ctr), C.byref(crec) if crec is not None else None)
            self._check(rc)
        res = SegmentResult(maps, tmin, npe, {n: int(getattr(ctr, n)) for n in COUNTER_NAMES})
        return (res, recs) if return_records else res

    # -- device-resident form (pointers are CUDA device addresses) -------------
    def run_photons_device(self, box, op, ro, tb, *, px, py, pz, pt, npos, n_photons, seed,
                           pid_offset=0, tau_ns, max_bounces=100_000, counts, first_ns,
                           counters, stream=None) -> None:
        ro = _as_readout(ro)
        rc = self.lib.cl_run_photons_device(
            self.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
            C.c_void_p(px), C.c_void_p(py), C.c_void_p(pz), C.c_void_p(pt) if pt else None,
            int(npos), int(n_photons), int(seed), int(pid_offset), float(np.float32(tau_ns)),
            int(max_bounces), C.c_void_p(counts), C.c_void_p(first_ns), C.c_void_p(counters),
            None, stream_arg(stream))
        self._check(rc)

    def run_segments_device(self, box, op, ro, tb, *, sx, sy, sz, st, src_offsets, src_segment,
                            n_src, n_segments, n_photons, seed, pid_offset=0, tau_ns,
                            max_bounces=100_000, maps, tmin, npe, counters, stream=None) -> None:
        ro = _as_readout(ro)
        rc = self.lib.cl_run_segments_device(
            self.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
            C.c_void_p(sx), C.c_void_p(sy), C.c_void_p(sz), C.c_void_p(st) if st else None,
            C.c_void_p(src_offsets), C.c_void_p(src_segment), int(n_src), int(n_segments),
            int(n_photons), int(seed), int(pid_offset), float(np.float32(tau_ns)), int(max_bounces),
            C.c_void_p(maps), C.c_void_p(tmin), C.c_void_p(npe), C.c_void_p(counters), None,
            stream_arg(stream))
        self._check(rc)

    def run_segments_moments_device(self, box, op, ro, tb, *, sx, sy, sz, st, src_offsets, src_segment,
                                    n_src, n_segments, n_photons, seed, pid_offset=0, tau_ns,
                                    max_bounces=100_000, maps, tmin, npe, counters, tsum, tsum2,
                                    stream=None) -> None:
        """run_segments_device plus fixed-point arrival-time sums per (segment, SiPM)."""
        ro = _as_readout(ro)
        rc = self.lib.cl_run_segments_moments_device(
            self.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
            C.c_void_p(sx), C.c_void_p(sy), C.c_void_p(sz), C.c_void_p(st) if st else None,
            C.c_void_p(src_offsets), C.c_void_p(src_segment), int(n_src), int(n_segments),
            int(n_photons), int(seed), int(pid_offset), float(np.float32(tau_ns)), int(max_bounces),
            C.c_void_p(maps), C.c_void_p(tmin), C.c_void_p(npe), C.c_void_p(counters),
            C.c_void_p(tsum), C.c_void_p(tsum2), stream_arg(stream))
        self._check(rc)

    def sync(self, stream=None) -> None:
        self._check(self.lib.cl_sync(self.handle, stream_arg(stream)))

    # -- diagnostics -----------------------------------------------------------
    def eval_math(self, fn: str, x: np.ndarray) -> np.ndarray:
        code = {"log": 0, "sin": 1, "cos": 2}[fn]
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty_like(x)
        self._check(self.lib.cl_debug_eval(self.handle, code, _ptr(x), _ptr(out), x.size, 0, 0))
        return out

    def log_table(self, n: int = 1 << 24) -> np.ndarray:
        """The transport's table of log((k+1) 2^-24), k < n (float32)."""
        out = np.empty(int(n), np.float32)
        self._check(self.lib.cl_debug_eval(self.handle, 6, None, _ptr(out), int(n), 0, 0))
        return out

    def philox(self, ctr: np.ndarray, seed: int, use_curand: bool = False) -> np.ndarray:
        ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
        out = np.empty_like(ctr)
        self._check(self.lib.cl_debug_eval(self.handle, 5 if use_curand else 3, _ptr(ctr),
                                           _ptr(out), ctr.shape[0], int(seed), 0))
        return out

    def randu_streams(self, seed: int, n_streams: int, n_per: int) -> np.ndarray:
        out = np.empty((n_streams, n_per), np.float32)
        self._check(self.lib.cl_debug_eval(self.handle, 4, None, _ptr(out), int(n_streams),
                                           int(seed), int(n_per)))
        return out


_default: Optional[Engine] = None
_default_lock = threading.Lock()


def default_engine() -> Engine:
    global _default
    with _default_lock:
        if _default is None:
            _default = Engine(0)
        return _default


def run_photons_ka(box, op, ro, tb, **kw):
    """run_photons_ka! on the default CUDA engine (device 0)."""
    return default_engine().run_photons_ka(box, op, ro, tb, **kw)


def run_photons(box, op, ro, tb, **kw):
    """run_photons! semantics, executed by the CUDA kernel."""
    return default_engine().run_photons(box, op, ro, tb, **kw)


def run_segments(box, op, ro, tb, **kw):
    return default_engine().run_segments(box, op, ro, tb, **kw)
