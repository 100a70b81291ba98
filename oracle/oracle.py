"""ctypes bindings of the CPU oracle (``oracle/build/libcl_oracle.so``).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

from crysplight_b200.params import (Accumulator, Box, Counters, OpticalParams, PhotonRecords,
                                    Readout, Records, TimeBinning, COUNTER_NAMES)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libcl_oracle.so")

_lock = threading.Lock()
_lib = None


class Stream(C.Structure):
    _fields_ = [("key", C.c_uint32 * 2), ("id_lo", C.c_uint32), ("id_hi", C.c_uint32),
                ("block", C.c_uint32), ("buf", C.c_uint32 * 4), ("i", C.c_int)]


class Photon(C.Structure):
    _fields_ = [("status", C.c_int32), ("idx", C.c_int16), ("t", C.c_float),
                ("bounces", C.c_int32), ("nscat", C.c_int32), ("steps", C.c_int32)]


class _Acc(C.Structure):
    _fields_ = [("counts", C.POINTER(C.c_uint32)), ("first_ns", C.POINTER(C.c_float)),
                ("c", Counters), ("nx", C.c_int32), ("ny", C.c_int32), ("nbins", C.c_int32)]


def build() -> str:
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            lib = C.CDLL(LIB_PATH)
            P, f, fp = C.c_void_p, C.c_float, C.POINTER(C.c_float)
            common = [C.POINTER(Box), C.POINTER(OpticalParams), C.POINTER(Readout),
                      C.POINTER(TimeBinning)]
            lib.or_philox4x32.argtypes = [P, P, P]
            lib.or_stream_init.argtypes = [C.POINTER(Stream), C.c_uint64, C.c_uint64]
            lib.or_next_u32.argtypes = [C.POINTER(Stream)]
            lib.or_next_u32.restype = C.c_uint32
            lib.or_randu.argtypes = [C.POINTER(Stream)]
            lib.or_randu.restype = f
            for n in ("or_logf", "or_sinf", "or_cosf"):
                getattr(lib, n).argtypes = [f]
                getattr(lib, n).restype = f
            lib.or_wall_hit.argtypes = [f, f, f, f, f, f, C.POINTER(Box), fp]
            lib.or_wall_hit.restype = C.c_int32
            lib.or_fresnel.argtypes = [f, f, f, fp]
            lib.or_fresnel.restype = C.c_int
            lib.or_isotropic_dir.argtypes = [C.POINTER(Stream), fp]
            lib.or_emission_time.argtypes = [C.POINTER(Stream), f]
            lib.or_emission_time.restype = f
            lib.or_gaussian.argtypes = [C.POINTER(Stream)]
            lib.or_gaussian.restype = f
            lib.or_lambertian_dir.argtypes = [C.POINTER(Stream), C.c_int32, fp]
            lib.or_rayleigh_dir.argtypes = [C.POINTER(Stream), fp, fp]
            lib.or_surface_interact.argtypes = [C.POINTER(Stream), fp, C.c_int32, f, f, fp]
            lib.or_surface_interact.restype = C.c_int
            lib.or_propagate_photon.argtypes = [C.POINTER(_Acc)] + common + [
                C.POINTER(Stream), f, f, f, f, f, f, f, C.c_int32, C.POINTER(Photon)]
            lib.or_propagate_photon.restype = C.c_int32
            lib.or_run_photons.argtypes = common + [P, P, P, C.c_int32, C.c_int64, C.c_uint64,
                                                    f, C.c_int32, C.c_int, P, P, C.POINTER(Counters)]
            lib.or_run_photons.restype = C.c_int
            lib.or_run_photons_ka.argtypes = common + [
                P, P, P, P, C.c_int32, C.c_int64, C.c_uint64, C.c_uint64, f, C.c_int32, C.c_int,
                P, P, C.POINTER(Counters), C.POINTER(Records), C.POINTER(C.c_int64)]
            lib.or_run_photons_ka.restype = C.c_int
            lib.or_run_segments.argtypes = common + [
                P, P, P, P, P, P, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, f, C.c_int32,
                C.c_int, P, P, P, C.POINTER(Counters), C.POINTER(Records), C.POINTER(C.c_int64)]
            lib.or_run_segments.restype = C.c_int
            lib.or_eval_batch.argtypes = [C.c_int, P, P, C.c_int64]
            lib.or_randu_batch.argtypes = [C.c_uint64, C.c_int64, C.c_int32, P]
            lib.or_philox_batch.argtypes = [P, C.c_uint64, C.c_int64, P]
            _lib = lib
        return _lib


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


# ---- primitives ----------------------------------------------------------------

def philox4x32(ctr, key) -> tuple:
    lib = load()
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) & 0xFFFFFFFF for v in key])
    o = (C.c_uint32 * 4)()
    lib.or_philox4x32(c, k, o)
    return tuple(o)


def philox_batch(ctr: np.ndarray, seed: int) -> np.ndarray:
    ctr = np.ascontiguousarray(ctr, dtype=np.uint32).reshape(-1, 4)
    out = np.empty_like(ctr)
    load().or_philox_batch(_p(ctr), int(seed), ctr.shape[0], _p(out))
    return out


def randu_streams(seed: int, n_streams: int, n_per: int) -> np.ndarray:
    out = np.empty((n_streams, n_per), np.float32)
    load().or_randu_batch(int(seed), int(n_streams), int(n_per), _p(out))
    return out


def eval_math(fn: str, x: np.ndarray) -> np.ndarray:
    code = {"log": 0, "sin": 1, "cos": 2}[fn]
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    load().or_eval_batch(code, _p(x), _p(out), x.size)
    return out


class PhiloxStream:
    """PhiloxStream(seed, photon_id), src/philox.jl:34-62."""

    def __init__(self, seed: int, photon_id: int):
        self.s = Stream()
        load().or_stream_init(C.byref(self.s), int(seed), int(photon_id))

    def next_u32(self) -> int:
        return load().or_next_u32(C.byref(self.s))

    def randu(self) -> float:
        return load().or_randu(C.byref(self.s))


def wall_hit(x, y, z, ux, uy, uz, box: Box):
    d = C.c_float()
    f = load().or_wall_hit(x, y, z, ux, uy, uz, C.byref(box), C.byref(d))
    return d.value, f


def fresnel(n1, n2, cosi):
    R = C.c_float()
    tir = load().or_fresnel(n1, n2, cosi, C.byref(R))
    return bool(tir), R.value


def isotropic_dir(s: PhiloxStream):
    u = (C.c_float * 3)()
    load().or_isotropic_dir(C.byref(s.s), u)
    return tuple(u)


def emission_time(s: PhiloxStream, tau):
    return load().or_emission_time(C.byref(s.s), tau)


def gaussian(s: PhiloxStream):
    return load().or_gaussian(C.byref(s.s))


def lambertian_dir(s: PhiloxStream, face: int):
    u = (C.c_float * 3)()
    load().or_lambertian_dir(C.byref(s.s), face, u)
    return tuple(u)


def rayleigh_dir(s: PhiloxStream, ux, uy, uz):
    u = (C.c_float * 3)(ux, uy, uz)
    v = (C.c_float * 3)()
    load().or_rayleigh_dir(C.byref(s.s), u, v)
    return tuple(v)


def surface_interact(s: PhiloxStream, ux, uy, uz, face, n_crystal, sigma_alpha):
    u = (C.c_float * 3)(ux, uy, uz)
    v = (C.c_float * 3)()
    tr = load().or_surface_interact(C.byref(s.s), u, face, n_crystal, sigma_alpha, v)
    return v[0], v[1], v[2], bool(tr)


class OracleAccumulator:
    """An Accumulator whose storage the C oracle writes into directly."""

    def __init__(self, grid, tb: TimeBinning):
        self.acc = Accumulator.empty(grid, tb)
        self._c = _Acc(self.acc.counts.ctypes.data_as(C.POINTER(C.c_uint32)),
                       self.acc.first_ns.ctypes.data_as(C.POINTER(C.c_float)), Counters(),
                       grid.nx, grid.ny, tb.nbins)

    def sync(self) -> Accumulator:
        self.acc.set_counters(self._c.c)
        return self.acc


def propagate_photon(acc: OracleAccumulator, box, op, ro, tb, s: PhiloxStream, x, y, z, ux, uy,
                     uz, t0, max_bounces=100_000):
    """propagate_photon!, src/transport.jl:118-234; returns (status, Photon record)."""
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    ph = Photon()
    st = load().or_propagate_photon(C.byref(acc._c) if acc is not None else None, C.byref(box),
                                    C.byref(op), C.byref(ro), C.byref(tb), C.byref(s.s), x, y, z,
                                    ux, uy, uz, t0, int(max_bounces), C.byref(ph))
    if acc is not None:
        acc.sync()
    return st, ph


# ---- drivers ---------------------------------------------------------------------

def _positions(pos, positions):
    if positions is None:
        positions = [pos]
    p = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
    return p, [np.ascontiguousarray(p[:, i]) for i in range(3)]


def run_photons(box, op, ro, tb, *, n_photons, seed, pos=None, positions=None, tau_ns,
                max_bounces=100_000, nthreads=None) -> Accumulator:
    """run_photons!, src/transport.jl:245-273 (threaded, static striping)."""
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    p, (px, py, pz) = _positions(pos, positions)
    acc = Accumulator.empty(ro.grid, tb)
    ctr = Counters()
    nt = nthreads or os.cpu_count() or 1
    rc = load().or_run_photons(C.byref(box), C.byref(op), C.byref(ro), C.byref(tb), _p(px), _p(py),
                               _p(pz), p.shape[0], int(n_photons), int(seed), float(np.float32(tau_ns)),
                               int(max_bounces), int(nt), _p(acc.counts), _p(acc.first_ns),
                               C.byref(ctr))
    if rc != 0:
        raise RuntimeError("oracle run_photons failed")
    acc.set_counters(ctr)
    return acc


def run_photons_ka(box, op, ro, tb, *, n_photons, seed, pos=None, positions=None, t0s=None,
                   pid_offset=0, tau_ns, max_bounces=100_000, return_records=False,
                   nthreads=None, return_steps=False):
    """transport_kernel! + run_photons_ka!'s host reduction, src/kernel.jl:159-367."""
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    p, (px, py, pz) = _positions(pos, positions)
    pt = None if t0s is None else np.ascontiguousarray(np.asarray(t0s, np.float32).reshape(-1))
    acc = Accumulator.empty(ro.grid, tb)
    ctr = Counters()
    recs = PhotonRecords.empty(int(n_photons)) if return_records else None
    steps = C.c_int64()
    nt = nthreads or os.cpu_count() or 1
    rc = load().or_run_photons_ka(
        C.byref(box), C.byref(op), C.byref(ro), C.byref(tb), _p(px), _p(py), _p(pz), _p(pt),
        p.shape[0], int(n_photons), int(seed), int(pid_offset), float(np.float32(tau_ns)),
        int(max_bounces), int(nt), _p(acc.counts), _p(acc.first_ns), C.byref(ctr),
        C.byref(recs.as_c()) if recs is not None else None, C.byref(steps))
    if rc != 0:
        raise RuntimeError("oracle run_photons_ka failed")
    acc.set_counters(ctr)
    out = (acc, recs) if return_records else acc
    return (out, steps.value) if return_steps else out


def run_segments(box, op, ro, tb, *, sources, photons_per_source, segment_of_source, n_segments,
                 seed, t0s=None, pid_offset=0, tau_ns, max_bounces=100_000, return_records=False,
                 nthreads=None, return_steps=False):
    """Per-segment reduction over records (src/events.jl:65-91, any layout)."""
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    s = np.ascontiguousarray(np.asarray(sources, np.float32).reshape(-1, 3))
    sx, sy, sz = (np.ascontiguousarray(s[:, i]) for i in range(3))
    cnt = np.asarray(photons_per_source, np.int64)
    off = np.zeros(s.shape[0] + 1, np.int64)
    np.cumsum(cnt, out=off[1:])
    seg = np.ascontiguousarray(np.asarray(segment_of_source, np.int32))
    st = None if t0s is None else np.ascontiguousarray(np.asarray(t0s, np.float32).reshape(-1))
    nx, ny = ro.grid.nx, ro.grid.ny
    maps = np.zeros((nx, ny, int(n_segments)), np.uint32, order="F")
    tmin = np.zeros((nx, ny, int(n_segments)), np.float32, order="F")
    npe = np.zeros(int(n_segments), np.int32)
    ctr = Counters()
    n = int(off[-1])
    recs = PhotonRecords.empty(n) if return_records else None
    steps = C.c_int64()
    nt = nthreads or os.cpu_count() or 1
    rc = load().or_run_segments(
        C.byref(box), C.byref(op), C.byref(ro), C.byref(tb), _p(sx), _p(sy), _p(sz), _p(st),
        _p(off), _p(seg), s.shape[0], int(n_segments), int(seed), int(pid_offset),
        float(np.float32(tau_ns)), int(max_bounces), int(nt), _p(maps), _p(tmin), _p(npe),
        C.byref(ctr), C.byref(recs.as_c()) if recs is not None else None, C.byref(steps))
    if rc != 0:
        raise RuntimeError("oracle run_segments failed")
    res = {"maps": maps, "tmin": tmin, "npe": npe,
           "counters": {k: int(getattr(ctr, k)) for k in COUNTER_NAMES}}
    out = (res, recs) if return_records else res
    return (out, steps.value) if return_steps else out
