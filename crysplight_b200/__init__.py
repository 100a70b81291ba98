"""crysplight_b200 — B200-native optical-photon transport engine for CryspLight.

The product is the sm_100a C-ABI library ``lib/libcrysplight_cuda.so``
(interface: ``include/crysplight_cuda.h``).  This package is its host-side
mirror of the reference's Julia API: the parameter structs, ``Accumulator``,
``run_photons_ka`` / ``run_photons`` / ``run_segments``, the run-TOML loader
and the output writers.
"""
from .params import (Accumulator, Box, Counters, OpticalParams, PhotonRecords, Readout,
                     SipmGrid, TimeBinning, FACE_BACK, FACE_FRONT, FACE_XM, FACE_XP,
                     FACE_YM, FACE_YP, STATUS_ABS_BULK, STATUS_ABS_SIPM, STATUS_ABS_SUR,
                     STATUS_ABS_WALL, STATUS_CAP, STATUS_DETECTED, surface_has_gap,
                     deg2rad_f32)
from .transport import (Engine, SegmentResult, default_engine, run_photons, run_photons_ka,
                        run_segments)

__all__ = [
    "Accumulator", "Box", "Counters", "OpticalParams", "PhotonRecords", "Readout", "SipmGrid",
    "TimeBinning", "Engine", "SegmentResult", "default_engine", "run_photons", "run_photons_ka",
    "run_segments", "surface_has_gap", "deg2rad_f32",
    "FACE_XP", "FACE_XM", "FACE_YP", "FACE_YM", "FACE_BACK", "FACE_FRONT",
    "STATUS_DETECTED", "STATUS_ABS_BULK", "STATUS_ABS_WALL", "STATUS_ABS_SIPM", "STATUS_CAP",
    "STATUS_ABS_SUR",
]
