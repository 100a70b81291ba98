"""Reference operations per photon-step, counted by the instrumented oracle.

TEST/ANALYSIS INFRASTRUCTURE.  The analysis build of the oracle
(``build/libcl_oracle_ops.so``, -DOR_COUNT_OPS) adds, at each expression of
the reference's transport (src/philox.jl, src/optics.jl, src/geometry.jl,
src/generation.jl, src/transport.jl), the number of Float32/integer
arithmetic operations it performs (log/sin/cos/sqrt/div count one each;
compares and selects are not counted).  Divided by the photon-steps of the
same run this gives the algorithmic operations per step used by the
transport's roofline.

    python -m oracle.opcount
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
OPS_LIB = os.path.join(HERE, "build", "libcl_oracle_ops.so")


def ops_per_step(box, op, ro, tb, *, n_photons, seed, pos=None, positions=None, tau_ns,
                 pid_offset=0, max_bounces=100_000):
    O.build()
    lib = C.CDLL(OPS_LIB)
    lib.or_ops_read.restype = C.c_uint64
    lib.or_ops_reset.restype = None
    lib.or_run_photons_ka.restype = C.c_int
    from crysplight_b200.params import Readout, Counters
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    if positions is None:
        positions = [pos]
    p = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    px, py, pz = (np.ascontiguousarray(p[:, i]) for i in range(3))
    steps = C.c_int64()
    lib.or_ops_reset()
    rc = lib.or_run_photons_ka(
        C.byref(box), C.byref(op), C.byref(ro), C.byref(tb), C.c_void_p(px.ctypes.data),
        C.c_void_p(py.ctypes.data), C.c_void_p(pz.ctypes.data), None, C.c_int32(p.shape[0]),
        C.c_int64(n_photons), C.c_uint64(seed), C.c_uint64(pid_offset), C.c_float(tau_ns),
        C.c_int32(max_bounces), C.c_int(1), None, None, None, None, C.byref(steps))
    assert rc == 0
    ops = lib.or_ops_read()
    return ops / steps.value, steps.value / n_photons


if __name__ == "__main__":
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from crysplight_b200.params import (Box, OpticalParams, Readout, SipmGrid, TimeBinning,
                                        deg2rad_f32)
    from crysplight_b200.scan import scan_points
    grid, tb = SipmGrid(6, 8, 8), TimeBinning(100, 80)
    c1 = OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, deg2rad_f32(1.3), 1.0)
    c2 = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, deg2rad_f32(1.3), 1.0)
    r1 = ops_per_step(Box((48, 48, 37.2)), c1, grid, tb, n_photons=200_000, seed=1234,
                      pos=(24, 24, 18.6), tau_ns=1000.0)
    pts = scan_points(256, Box((48, 48, 22.4)), 7)
    tot_ops = tot_steps = 0.0
    for pidx in range(0, 256, 16):
        o, sp = ops_per_step(Box((48, 48, 22.4)), c2, grid, tb, n_photons=20_000, seed=1234,
                             pos=tuple(pts[pidx]), pid_offset=pidx * 200_000, tau_ns=1768.0)
        tot_ops += o * sp * 20_000
        tot_steps += sp * 20_000
    print(f"CsI(Tl)+Teflon point source (centre): {r1[0]:.1f} ops/step, {r1[1]:.2f} steps/photon")
    print(f"BGO+ESR scan (16 of 256 points): {tot_ops / tot_steps:.1f} ops/step, "
          f"{tot_steps / (16 * 20_000):.2f} steps/photon")
