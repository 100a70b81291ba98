"""511 keV gamma events: gamma stage on the host, optical transport on the GPU.

Mirrors CryspLight's event pipeline ``run_events!`` (src/events.jl:39-125):
per event, a 511 keV gamma enters the front face (z = 0) at a uniform (x, y)
along +z; its energy deposits (the reference's vendored gamma core, restated
in C in ``csrc/cl_gamma.cpp``) each emit Poisson(yield * E) photons from the
deposit point, delayed by the deposit time; all photons of all events are
transported in one launch over prefix-summed photon offsets
(``cl_run_segments``), and each event's detections are reduced into its 8x8
map, first-hit times and photoelectron count.

Photon ids follow the reference: the global running photon index (1-based,
event-major, deposit order), so the optical stage of an event is bit-exact
given its deposits.  The gamma stage draws from its own Philox stream per
event (the reference's Julia Xoshiro stream cannot be reproduced here), so
event-level results agree with the reference statistically.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from .params import Box, OpticalParams, Readout, TimeBinning
from .config import PKG_DATA_DIR

DEP_PHOTO, DEP_COMPTON, DEP_BELOWCUT = 0, 1, 2      # src/gamma_interface.jl:11-13


def load_xcom(path: str) -> dict:
    """NIST XCOM table (src/gamma/nist_data.jl:19-35): rows of 8 numeric columns
    (E, coherent, incoherent, photoelectric, pair nuclear, pair electron,
    total with / without coherent), mu/rho in cm^2/g; other lines skipped."""
    rows = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or not ("0" <= s[0] <= "9"):
                continue
            fields = s.split()
            if len(fields) < 8:
                continue
            rows.append([float(v) for v in fields[:8]])
    if not rows:
        raise ValueError(f"no XCOM data rows in {path}")
    m = np.asarray(rows, dtype=np.float64)
    keys = ("E_MeV", "coherent", "incoherent", "photoelectric", "pair_nuclear",
            "pair_electron", "total_w_coh", "total_no_coh")
    return {k: np.ascontiguousarray(m[:, i]) for i, k in enumerate(keys)}


def _declare(lib):
    if getattr(lib, "_gamma_declared", False):
        return
    P = C.c_void_p
    lib.cl_gamma_material_create.argtypes = [C.POINTER(C.c_void_p), P, P, P, P, P, C.c_int32,
                                             C.c_double]
    lib.cl_gamma_material_create.restype = C.c_int
    lib.cl_gamma_material_destroy.argtypes = [P]
    lib.cl_gamma_material_destroy.restype = None
    lib.cl_gamma_last_error.restype = C.c_char_p
    lib.cl_gamma_sigma.argtypes = [P, C.c_double, P]
    lib.cl_gamma_sigma.restype = C.c_int
    lib.cl_gamma_deposits.argtypes = [P, C.POINTER(Box), P, P, C.c_double, C.c_uint64, C.c_uint64,
                                      P, C.c_int32, C.POINTER(C.c_int32)]
    lib.cl_gamma_deposits.restype = C.c_int
    lib.cl_rand_poisson.argtypes = [C.c_uint64, C.c_uint64, C.c_double]
    lib.cl_rand_poisson.restype = C.c_int64
    lib.cl_gamma_events.argtypes = [P, C.POINTER(Box), C.c_int64, C.c_int64, C.c_uint64, C.c_double,
                                    C.c_double, C.c_int, P, P, P, P, P, P, P, P, C.c_int64, P, P, P,
                                    P, C.POINTER(C.c_int64)]
    lib.cl_gamma_events.restype = C.c_int
    lib._gamma_declared = True


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class GammaMaterial:
    """Gamma.make_material(name, density, xcom_csv) (src/gamma/gmaterials.jl:22-31)."""

    def __init__(self, name: str, density: float, xcom: Optional[dict]):
        self.lib = _lib.load()
        _declare(self.lib)
        self.name = name
        self.density = float(density)
        h = C.c_void_p()
        if xcom is None:
            rc = self.lib.cl_gamma_material_create(C.byref(h), None, None, None, None, None, 0, 0.0)
        else:
            cols = [np.ascontiguousarray(xcom[k], dtype=np.float64) for k in
                    ("E_MeV", "incoherent", "photoelectric", "pair_nuclear", "pair_electron")]
            self._cols = cols
            rc = self.lib.cl_gamma_material_create(C.byref(h), *[_p(c) for c in cols],
                                                   int(cols[0].size), self.density)
        if rc != 0:
            raise ValueError(self.lib.cl_gamma_last_error().decode())
        self.handle = h

    @classmethod
    def from_csv(cls, name: str, density: float, path: str) -> "GammaMaterial":
        if not os.path.isabs(path) and not os.path.exists(path):
            path = os.path.join(PKG_DATA_DIR, path)
        return cls(name, density, load_xcom(path))

    @classmethod
    def vacuum(cls) -> "GammaMaterial":
        """vacuum_material() (src/gamma/gmaterials.jl:34-36)."""
        return cls("Vacuum", 0.0, None)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self.lib.cl_gamma_material_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def sigma_macro(self, E_MeV: float) -> tuple:
        out = np.zeros(3, np.float64)
        self.lib.cl_gamma_sigma(self.handle, float(E_MeV), _p(out))
        return tuple(float(v) for v in out)

    def mfp(self, E_MeV: float) -> float:
        """mfp (src/gamma/gmaterials.jl:59-61): mean free path in cm."""
        s = sum(self.sigma_macro(E_MeV))
        return 1.0 / s if s > 0 else float("inf")


def gamma_deposits(mat: GammaMaterial, box: Box, entry_mm, direction=(0.0, 0.0, 1.0), *,
                   seed: int, stream: int, e0_mev: float = 0.511) -> list:
    """gamma_deposits (src/gamma_interface.jl:30-49): [(x, y, z, E_keV, t_ns, proc), ...]."""
    lib = mat.lib
    entry = np.asarray(entry_mm, np.float32)
    d = np.asarray(direction, np.float64)
    out = np.zeros((256, 6), np.float32)
    n = C.c_int32()
    rc = lib.cl_gamma_deposits(mat.handle, C.byref(box), _p(entry), _p(d), float(e0_mev), int(seed),
                               int(stream), _p(out), 256, C.byref(n))
    if rc != 0:
        raise RuntimeError(lib.cl_gamma_last_error().decode())
    return [tuple(float(v) for v in out[i, :5]) + (int(out[i, 5]),) for i in range(n.value)]


def rand_poisson(seed: int, stream: int, lam: float) -> int:
    """rand_poisson (src/events.jl:11-22) on stream `stream` of `seed`."""
    lib = _lib.load()
    _declare(lib)
    return int(lib.cl_rand_poisson(int(seed), int(stream), float(lam)))


@dataclass
class GammaStage:
    """Output of the host gamma stage for a block of events."""
    edep: np.ndarray
    xyz1: np.ndarray
    e1: np.ndarray
    xyz2: np.ndarray
    e2: np.ndarray
    er: np.ndarray
    int_type: np.ndarray
    n_int: np.ndarray
    dep_xyz: np.ndarray        # (n_dep, 3) float32
    dep_t: np.ndarray          # (n_dep,) float32
    dep_event: np.ndarray      # (n_dep,) int32, event index within the block
    dep_photons: np.ndarray    # (n_dep,) int64

    @property
    def n_photons(self) -> int:
        return int(self.dep_photons.sum())


def gamma_stage(mat: GammaMaterial, box: Box, *, n_events: int, seed: int, yield_per_mev: float,
                e0_mev: float = 0.511, ev0: int = 0, nthreads: int = 0) -> GammaStage:
    lib = mat.lib
    n = int(n_events)
    edep = np.zeros(n, np.float32)
    xyz1 = np.zeros((3, n), np.float32, order="F")
    e1 = np.zeros(n, np.float32)
    xyz2 = np.zeros((3, n), np.float32, order="F")
    e2 = np.zeros(n, np.float32)
    er = np.zeros(n, np.float32)
    int_type = np.zeros(n, np.int8)
    n_int = np.zeros(n, np.int16)
    cap = max(16, 8 * n)
    while True:
        dep_xyz = np.zeros((cap, 3), np.float32)
        dep_t = np.zeros(cap, np.float32)
        dep_ev = np.zeros(cap, np.int32)
        dep_ph = np.zeros(cap, np.int64)
        nd = C.c_int64()
        rc = lib.cl_gamma_events(mat.handle, C.byref(box), int(ev0), n, int(seed), float(e0_mev),
                                 float(yield_per_mev), int(nthreads), _p(edep), _p(xyz1), _p(e1),
                                 _p(xyz2), _p(e2), _p(er), _p(int_type), _p(n_int), cap,
                                 _p(dep_xyz), _p(dep_t), _p(dep_ev), _p(dep_ph), C.byref(nd))
        if rc == 0:
            break
        if nd.value > cap:
            cap = int(nd.value)
            continue
        raise RuntimeError(lib.cl_gamma_last_error().decode())
    k = nd.value
    return GammaStage(edep, xyz1, e1, xyz2, e2, er, int_type, n_int, dep_xyz[:k], dep_t[:k],
                      dep_ev[:k], dep_ph[:k])


@dataclass
class EventsResult:
    """run_events! result (src/events.jl:122-124), Julia column-major shapes."""
    edep: np.ndarray           # (n,) float32 keV
    npe: np.ndarray            # (n,) int32
    maps: np.ndarray           # (nx, ny, n) uint16, Fortran order
    tmin: np.ndarray           # (nx, ny, n) float32, +Inf where no hit
    xyz1: np.ndarray           # (3, n) float32 mm
    e1: np.ndarray
    xyz2: np.ndarray
    e2: np.ndarray
    er: np.ndarray
    int_type: np.ndarray       # int8: -1 none, 0 photoelectric, X >= 1 Compton scatters
    n_int: np.ndarray          # int16
    n_photons: int = 0
    counters: Optional[dict] = None


def run_events(box: Box, op: OpticalParams, ro, tb: TimeBinning, material: GammaMaterial,
               yield_per_mev: float, *, n_events: int, seed: int, tau_ns: float,
               e0_mev: float = 0.511, max_bounces: int = 100_000, engine=None,
               batch_events: Optional[int] = None, nthreads: int = 0) -> EventsResult:
    """run_events! (src/events.jl:39-125) with the optical stage on the GPU.

    All events go through one transport launch per batch of ``batch_events``
    events (default: all at once); photon ids continue across batches as the
    reference's ``pid_offset`` does."""
    from .transport import default_engine
    eng = engine or default_engine()
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    n = int(n_events)
    nx, ny = ro.grid.nx, ro.grid.ny
    out = EventsResult(np.zeros(n, np.float32), np.zeros(n, np.int32),
                       np.zeros((nx, ny, n), np.uint16, order="F"),
                       np.full((nx, ny, n), np.inf, np.float32, order="F"),
                       np.zeros((3, n), np.float32, order="F"), np.zeros(n, np.float32),
                       np.zeros((3, n), np.float32, order="F"), np.zeros(n, np.float32),
                       np.zeros(n, np.float32), np.full(n, -1, np.int8), np.zeros(n, np.int16))
    counters = None
    pid0 = 0
    step = int(batch_events or n or 1)
    for b0 in range(0, n, step):
        nb = min(step, n - b0)
        g = gamma_stage(material, box, n_events=nb, seed=seed, yield_per_mev=yield_per_mev,
                        e0_mev=e0_mev, ev0=b0, nthreads=nthreads)
        sl = slice(b0, b0 + nb)
        out.edep[sl] = g.edep; out.e1[sl] = g.e1; out.e2[sl] = g.e2; out.er[sl] = g.er
        out.xyz1[:, sl] = g.xyz1; out.xyz2[:, sl] = g.xyz2
        out.int_type[sl] = g.int_type; out.n_int[sl] = g.n_int
        if g.dep_photons.size == 0 or g.n_photons == 0:
            continue
        res = eng.run_segments(box, op, ro, tb, sources=g.dep_xyz, photons_per_source=g.dep_photons,
                               segment_of_source=g.dep_event, n_segments=nb, seed=seed,
                               t0s=g.dep_t, pid_offset=pid0, tau_ns=tau_ns,
                               max_bounces=max_bounces)
        pid0 += g.n_photons
        out.maps[:, :, sl] = (res.maps & 0xFFFF).astype(np.uint16)   # UInt16 maps wrap as in Julia
        out.tmin[:, :, sl] = res.tmin
        out.npe[sl] = res.npe
        if counters is None:
            counters = dict(res.counters)
        else:
            for k, v in res.counters.items():
                counters[k] += v
    out.n_photons = pid0
    out.counters = counters
    return out
