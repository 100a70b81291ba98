"""The C-ABI library loads and exports every symbol include/*.h declares, and
its struct layouts match the reference's Julia isbits structs.  No GPU."""
import ctypes as C
import glob
import os
import re

import pytest

from crysplight_b200 import _lib
from crysplight_b200.params import (Box, Counters, OpticalParams, Readout, Records, SipmGrid,
                                    TimeBinning)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(cl_[a-z_0-9]+)\s*\(", src):
            if m.group(1) not in names:
                names.append(m.group(1))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        from crysplight_b200 import build
        build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 13
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(names)


def test_version(lib):
    assert lib.cl_abi_version() == 1
    assert b"sm_100a" in lib.cl_version()


def test_struct_layouts_match_julia_isbits():
    # OpticalParams: 5 x Float32, 2 x Bool, (pad), 2 x Float32 -> 32 bytes
    assert C.sizeof(OpticalParams) == 32
    assert OpticalParams.sigma_alpha.offset == 24 and OpticalParams.pde.offset == 28
    assert C.sizeof(SipmGrid) == 12
    # Readout: grid(12) disc@12 cx@16 cy@20 r2@24 sur_R@28 sur_specular@32 two_sided@33 -> 36
    assert C.sizeof(Readout) == 36
    assert Readout.cx.offset == 16 and Readout.sur_specular.offset == 32
    assert Readout.two_sided.offset == 33
    assert C.sizeof(TimeBinning) == 8 and C.sizeof(Box) == 12
    assert C.sizeof(Counters) == 72 and C.sizeof(Records) == 32


def test_errors_without_device_are_reported_not_fatal(lib):
    """cl_create on a machine without a usable GPU returns an error code and a
    message instead of aborting (the product never falls back to the CPU)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    h = C.c_void_p()
    rc = lib.cl_create(C.byref(h), 0)
    assert rc < 0
    assert lib.cl_last_error(None)
    # null handle is rejected
    assert lib.cl_sync(None, None) == _lib.CL_ERR_STATE


def test_readout_keyword_constructor():
    ro = Readout(SipmGrid(6, 8, 8), center=(24, 24), radius=10, sur_R=0.95, sur_specular=True)
    assert ro.disc == 1 and ro.r2 == pytest.approx(100.0) and ro.sur_specular == 1
    ro = Readout(SipmGrid(6, 8, 8), two_sided=True)
    assert ro.disc == 0 and ro.two_sided == 1
