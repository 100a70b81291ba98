"""Emission-point scans: the per-point workload of the BGO + ESR sweep.

The reference has no point generator; this one is defined here.  Point p of a
scan with seed s is (u0 * Lx, u1 * Ly, u2 * Lz) in Float32, where (u0, u1, u2)
are the first three outputs of Philox4x32-10 with key (s lo, s hi) and counter
(p, 0, 0, 0), each mapped to (0, 1] by ((x >> 8) + 1) * 2^-24 as in
src/philox.jl:62.  Each point then emits its own photons with pid offset
(photons before it), exactly as one run_photons_ka!(...; pos, pid_offset)
call per point would.
"""
from __future__ import annotations

import numpy as np

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, seed: int) -> np.ndarray:
    """Vectorised Philox4x32-10 (src/philox.jl:10-28): ctr (n, 4) uint32 -> (n, 4)."""
    c = np.asarray(ctr, dtype=np.uint64).reshape(-1, 4).copy()
    k0 = np.uint64(seed & 0xFFFFFFFF)
    k1 = np.uint64((seed >> 32) & 0xFFFFFFFF)
    c0, c1, c2, c3 = c[:, 0], c[:, 1], c[:, 2], c[:, 3]
    for r in range(10):
        p0 = _M0 * c0
        p1 = _M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c0, c1, c2, c3 = hi1 ^ c1 ^ k0, lo1, hi0 ^ c3 ^ k1, lo0
        if r < 9:
            k0 = (k0 + _W0) & _MASK
            k1 = (k1 + _W1) & _MASK
    return np.stack([c0, c1, c2, c3], axis=1).astype(np.uint32)


def u32_to_randu(x: np.ndarray) -> np.ndarray:
    """((x >>> 8) + 1.0f0) * 2^-24 in Float32 (exact)."""
    return ((np.asarray(x, np.uint32) >> np.uint32(8)).astype(np.float32) + np.float32(1.0)) \
        * np.float32(2.0 ** -24)


def scan_points(n_points: int, box, seed: int = 7) -> np.ndarray:
    """(n_points, 3) float32 emission points uniform in the box."""
    ctr = np.zeros((n_points, 4), np.uint32)
    ctr[:, 0] = np.arange(n_points, dtype=np.uint32)
    u = u32_to_randu(philox4x32_10(ctr, seed)[:, :3])
    L = np.asarray(tuple(box.L), dtype=np.float32)
    return (u * L[None, :]).astype(np.float32)
