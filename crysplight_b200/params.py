"""Parameter structs of the transport call, mirroring CryspLight's Julia types.

The ctypes layouts match the C-ABI of ``include/crysplight_cuda.h``, which in
turn matches the Julia isbits structs (C alignment, ``Bool`` = ``uint8``):

* ``Box``            src/geometry.jl:14-16
* ``OpticalParams``  src/transport.jl:14-24
* ``SipmGrid``       src/transport.jl:26-30
* ``Readout``        src/transport.jl:41-57 (keyword constructor included)
* ``TimeBinning``    src/transport.jl:59-62
* ``Accumulator``    src/transport.jl:64-94 (``merge``, ``total_terminated``)

Arrays follow Julia's column-major layout: ``Accumulator.counts`` is a numpy
array of shape (nx, ny, nbins+1) in Fortran order, so ``counts[i, j, b]`` is
Julia's ``counts[i+1, j+1, b+1]``.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

# Face codes, src/geometry.jl:6-11
FACE_XP, FACE_XM, FACE_YP, FACE_YM, FACE_BACK, FACE_FRONT = 1, 2, 3, 4, 5, 6

# Photon fates, src/transport.jl:6-12
STATUS_DETECTED = 1
STATUS_ABS_BULK = 2
STATUS_ABS_WALL = 3
STATUS_ABS_SIPM = 4
STATUS_CAP = 5
STATUS_ABS_SUR = 6

C_MM_NS = 299.792458


def f32(x) -> float:
    """Round a Python number to Float32 (Julia's ``Float32(x)``)."""
    return float(np.float32(x))


class Box(C.Structure):
    _fields_ = [("L", C.c_float * 3)]

    def __init__(self, L=(48.0, 48.0, 37.2)):
        super().__init__()
        for i in range(3):
            self.L[i] = f32(L[i])

    @property
    def size(self):
        return tuple(self.L)

    def __repr__(self):
        return f"Box({tuple(self.L)})"


class OpticalParams(C.Structure):
    _fields_ = [
        ("n_crystal", C.c_float),
        ("n_coupling", C.c_float),
        ("abs_len_mm", C.c_float),
        ("rayleigh_mm", C.c_float),
        ("wrap_R", C.c_float),
        ("wrap_specular", C.c_uint8),
        ("air_gap", C.c_uint8),
        ("sigma_alpha", C.c_float),
        ("pde", C.c_float),
    ]

    def __init__(self, n_crystal, n_coupling, abs_len_mm, rayleigh_mm, wrap_R,
                 wrap_specular, air_gap, sigma_alpha, pde):
        super().__init__(f32(n_crystal), f32(n_coupling), f32(abs_len_mm), f32(rayleigh_mm),
                         f32(wrap_R), 1 if wrap_specular else 0, 1 if air_gap else 0,
                         f32(sigma_alpha), f32(pde))

    def __repr__(self):
        return ("OpticalParams(" + ", ".join(f"{n}={getattr(self, n)!r}" for n, _ in self._fields_) + ")")


class SipmGrid(C.Structure):
    _fields_ = [("pitch_mm", C.c_float), ("nx", C.c_int32), ("ny", C.c_int32)]

    def __init__(self, pitch_mm=6.0, nx=8, ny=8):
        super().__init__(f32(pitch_mm), int(nx), int(ny))


class Readout(C.Structure):
    """Readout of the z = Lz face (src/transport.jl:32-57).

    ``Readout(grid)`` is the full active face; ``Readout(grid, center=(cx, cy),
    radius=r, sur_R=..., sur_specular=..., two_sided=...)`` the disc aperture,
    exactly as the reference's keyword constructor.
    """
    _fields_ = [
        ("grid", SipmGrid),
        ("disc", C.c_uint8),
        ("cx", C.c_float),
        ("cy", C.c_float),
        ("r2", C.c_float),
        ("sur_R", C.c_float),
        ("sur_specular", C.c_uint8),
        ("two_sided", C.c_uint8),
    ]

    def __init__(self, grid: SipmGrid | None = None, *, center=None, radius=None, sur_R=0,
                 sur_specular: bool = False, two_sided: bool = False):
        grid = grid if grid is not None else SipmGrid()
        if radius is None:
            super().__init__(grid, 0, 0.0, 0.0, 0.0, 0.0, 0, 1 if two_sided else 0)
        else:
            r = np.float32(radius)
            super().__init__(grid, 1, f32(center[0]), f32(center[1]), float(r * r),
                             f32(sur_R), 1 if sur_specular else 0, 1 if two_sided else 0)


class TimeBinning(C.Structure):
    _fields_ = [("bin_ns", C.c_float), ("nbins", C.c_int32)]

    def __init__(self, bin_ns=100.0, nbins=80):
        super().__init__(f32(bin_ns), int(nbins))


class Counters(C.Structure):
    """Scalar fields of Accumulator in the reference's order."""
    _fields_ = [(n, C.c_int64) for n in (
        "ndet", "ndet_front", "nabs_bulk", "nabs_wall", "nabs_sipm", "ncap",
        "nabs_sur", "nscat", "sum_bounces_det")]


class Records(C.Structure):
    """Pointers to per-photon records (cl_records)."""
    _fields_ = [
        ("status", C.POINTER(C.c_uint8)),
        ("idx", C.POINTER(C.c_int16)),
        ("t", C.POINTER(C.c_float)),
        ("bounces", C.POINTER(C.c_int32)),
    ]


COUNTER_NAMES = tuple(n for n, _ in Counters._fields_)


@dataclass
class PhotonRecords:
    """Per-photon records of transport_kernel! (src/kernel.jl:300-303)."""
    status: np.ndarray
    idx: np.ndarray
    t: np.ndarray
    bounces: np.ndarray

    @classmethod
    def empty(cls, n: int) -> "PhotonRecords":
        return cls(np.zeros(n, np.uint8), np.zeros(n, np.int16),
                   np.zeros(n, np.float32), np.zeros(n, np.int32))

    def as_c(self) -> Records:
        return Records(self.status.ctypes.data_as(C.POINTER(C.c_uint8)),
                       self.idx.ctypes.data_as(C.POINTER(C.c_int16)),
                       self.t.ctypes.data_as(C.POINTER(C.c_float)),
                       self.bounces.ctypes.data_as(C.POINTER(C.c_int32)))


@dataclass
class Accumulator:
    """Counts, first detection times and fate counters (src/transport.jl:64-94)."""
    counts: np.ndarray                       # (nx, ny, nbins+1) uint32, Fortran order
    first_ns: np.ndarray                     # (nx, ny) float32, Fortran order, +Inf if none
    ndet: int = 0
    ndet_front: int = 0
    nabs_bulk: int = 0
    nabs_wall: int = 0
    nabs_sipm: int = 0
    ncap: int = 0
    nabs_sur: int = 0
    nscat: int = 0
    sum_bounces_det: int = 0

    @classmethod
    def empty(cls, grid: SipmGrid, tb: TimeBinning) -> "Accumulator":
        return cls(np.zeros((grid.nx, grid.ny, tb.nbins + 1), np.uint32, order="F"),
                   np.full((grid.nx, grid.ny), np.inf, np.float32, order="F"))

    def set_counters(self, c: Counters) -> None:
        for n in COUNTER_NAMES:
            setattr(self, n, int(getattr(c, n)))

    def counters(self) -> dict:
        return {n: getattr(self, n) for n in COUNTER_NAMES}

    def total_terminated(self) -> int:
        """total_terminated, src/transport.jl:93-94."""
        return (self.ndet + self.nabs_bulk + self.nabs_wall + self.nabs_sipm
                + self.ncap + self.nabs_sur)

    def merge(self, other: "Accumulator") -> "Accumulator":
        """merge!, src/transport.jl:82-91."""
        self.counts += other.counts
        np.minimum(self.first_ns, other.first_ns, out=self.first_ns)
        for n in COUNTER_NAMES:
            setattr(self, n, getattr(self, n) + getattr(other, n))
        return self


def surface_has_gap(finish: str) -> bool:
    """src/config.jl:22-25: validate a surface finish; True for back-painted."""
    if finish not in ("backpainted", "frontpainted"):
        raise ValueError(f"unknown finish: {finish}")
    return finish == "backpainted"


def deg2rad_f32(deg: float) -> float:
    """``Float32(deg2rad(x))`` with the conversion in Float64 (src/config.jl:49)."""
    return f32(float(deg) * (math.pi / 180.0))
