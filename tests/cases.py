"""Parameter sets shared by the tests (values from CryspLight's test suite,
test/runtests.jl, and its run files runs/point_csitl_teflon.toml,
runs/point_bgo_esr.toml)."""
import math

import numpy as np

from crysplight_b200.params import (Box, OpticalParams, Readout, SipmGrid, TimeBinning,
                                    deg2rad_f32)

INF = float("inf")
GRID = SipmGrid(6.0, 8, 8)            # test/runtests.jl:8
TB = TimeBinning(100.0, 40)           # test/runtests.jl:9
TB80 = TimeBinning(100.0, 80)
BOX_CSI = Box((48.0, 48.0, 37.2))
BOX_BGO = Box((48.0, 48.0, 22.4))
CENTRE_CSI = (24.0, 24.0, 18.6)
CENTRE_BGO = (24.0, 24.0, 11.2)


def ideal(n_crystal, *, wrap_R=1.0, spec=False, abs_len=INF, ray=INF, gap=True, sigma=0.0,
          pde=1.0):
    """test/runtests.jl:17-21."""
    return OpticalParams(n_crystal, 1.45, abs_len, ray, wrap_R, spec, gap, sigma, pde)


# CsI(Tl) + Teflon, PDE 1 (runs/point_csitl_teflon.toml + data/*.toml)
OP_CSI_TEFLON = OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, deg2rad_f32(1.3), 1.0)
TAU_CSI = 1000.0
# BGO + ESR, PDE 1 (runs/point_bgo_esr.toml + data/bgo.toml, data/esr.toml)
OP_BGO_ESR = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, deg2rad_f32(1.3), 1.0)
TAU_BGO = 1768.0
# every process at once (test/runtests.jl:168-170, 229-231)
OP_ALL = OpticalParams(1.95, 1.45, 500.0, 400.0, 0.98, False, True, deg2rad_f32(6.0), 0.4)
RO_ALL = Readout(GRID, center=(24, 24), radius=20, sur_R=0.9)
# cold-CsI benchmark configuration (scripts/bench_metal.jl:8-13)
OP_BENCH = OpticalParams(1.95, 1.45, 3000.0, 333.3, 0.99, False, True, deg2rad_f32(1.3), 1.0)


def scan_points(n_points: int, box: Box, seed: int = 7):
    """Emission points uniform in the crystal: Philox key = seed, counter =
    (point index, 0, 0, 0); three uniforms ((x >> 8) + 1) * 2^-24 scaled by
    the box size.  This generator is defined by this project (the reference
    has none); it is the 256-point sweep of the BGO + ESR workload."""
    from crysplight_b200.scan import scan_points as sp
    return sp(n_points, box, seed)
