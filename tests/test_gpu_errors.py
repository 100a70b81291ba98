"""Argument errors of the device entry points come back as CL_ERR_ARG with a
message and leave the handle usable (the reference raises exceptions,
src/config.jl:23,59); nothing is launched for a rejected call."""
import ctypes as C

import numpy as np
import pytest

from cases import BOX_BGO, GRID, OP_BGO_ESR, TB80

pytestmark = pytest.mark.gpu


def test_events_surrogate_rejects_bad_arguments(engine):
    from crysplight_b200 import _lib
    from crysplight_b200.params import Readout
    lib = _lib.load()
    P = C.c_void_p
    ro = Readout(GRID)

    def call(**over):
        a = dict(n_src=0, n_photons=0, n_sites=0, n_segments=1, maps=1, tmin=1, npe=1, ctr=1, sx=None)
        a.update(over)
        return lib.cl_run_events_surrogate_device(
            engine.handle, C.byref(BOX_BGO), C.byref(OP_BGO_ESR), C.byref(ro), C.byref(TB80),
            P(a["sx"]) if a["sx"] else None, None, None, None, None, None, a["n_src"], a["n_photons"],
            1, 0, 1768.0, 100000, None, None, None, None, None, None, None, a["n_sites"], 2,
            a["n_segments"], P(a["maps"]), P(a["tmin"]), P(a["npe"]), P(a["ctr"]), None, None)
    assert call(n_segments=0) == _lib.CL_ERR_ARG
    assert b"n_segments" in lib.cl_last_error(engine.handle)
    assert call(n_photons=5) == _lib.CL_ERR_ARG                     # photons without sources
    assert call(n_src=3) == _lib.CL_ERR_ARG                         # null source arrays
    assert call(n_sites=4) == _lib.CL_ERR_ARG                       # null site arrays
    assert call(maps=0) == _lib.CL_ERR_ARG
    # the handle still works
    res = engine.run_segments(BOX_BGO, OP_BGO_ESR, GRID, TB80, sources=[(24.0, 24.0, 11.2)], photons_per_source=[500],
                              segment_of_source=[0], n_segments=1, seed=1, tau_ns=0.0)
    assert res.counters["ndet"] + res.counters["nabs_bulk"] + res.counters["nabs_wall"] + \
        res.counters["nabs_sipm"] + res.counters["ncap"] == 500


def test_combine_rejects_bad_arguments():
    from crysplight_b200 import _lib
    from crysplight_b200.params import Readout, SipmGrid
    lib = _lib.load()
    P = C.c_void_p
    args = lambda ro, pde, members=5, n=10: (P(1), members, n, P(1), P(1), P(1), C.byref(BOX_BGO), C.byref(ro),
                                             pde, 0.02, 1.0, P(1), P(1), P(1), P(1), P(1), None)
    assert lib.cl_surrogate_combine(*args(Readout(SipmGrid(6.0, 4, 4)), 0.4)) == _lib.CL_ERR_ARG   # 16 cells
    assert lib.cl_surrogate_combine(*args(Readout(GRID), 1.5)) == _lib.CL_ERR_ARG                   # PDE > 1
    assert lib.cl_surrogate_combine(*args(Readout(GRID), 0.4, members=0)) == _lib.CL_ERR_ARG
    assert lib.cl_surrogate_combine(*args(Readout(GRID), 0.4, n=0)) == _lib.CL_OK                    # nothing to do


def test_mlp_rejects_bad_batches():
    from crysplight_b200.surrogate import MLP
    from crysplight_b200._lib import CudaTransportError
    m = MLP(0, max_batch=1024, seed=0)
    try:
        import torch
        x = torch.zeros(100, 3, device="cuda")
        t = torch.zeros(100, 192, device="cuda")
        m.set_data(x, t)
        with pytest.raises(CudaTransportError):
            m.train(1, batch=100)          # not a multiple of 128
        with pytest.raises(CudaTransportError):
            m.train(1, batch=2048)         # above max_batch
        assert np.isfinite(m.train(2, batch=128))
    finally:
        m.close()


def test_sampled_site_with_a_bad_segment_is_skipped_and_reported(engine):
    """A device-side segment id outside the maps is caught in the sampler
    kernel (no out-of-range write) and reported by the sync."""
    import torch
    from crysplight_b200 import _lib
    from crysplight_b200.fast_events import SiteLight, sample_sites
    from crysplight_b200._lib import CudaTransportError
    n = 4
    xyz = torch.full((n, 3), 10.0, device="cuda")
    t0 = torch.zeros(n, device="cuda")
    ph = torch.full((n,), 1000, dtype=torch.int64, device="cuda")
    seg = torch.tensor([0, 1, 7, 1], dtype=torch.int32, device="cuda")      # 7 >= n_segments
    p = torch.full((n, 64), 0.004, device="cuda")
    light = SiteLight(p, torch.full((n, 64), 2.0, device="cuda"), torch.full((n, 64), 0.5, device="cuda"),
                      torch.zeros(n, device="cuda"), torch.zeros(n, dtype=torch.uint8, device="cuda"))
    with pytest.raises(CudaTransportError) as e:
        sample_sites(engine, BOX_BGO, OP_BGO_ESR, GRID, TB80, xyz=xyz, t0=t0, photons=ph, segment=seg,
                     n_segments=2, seed=3, tau_ns=1768.0, light=light)
    assert e.value.code == _lib.CL_ERR_ARG and b"segment" in engine.lib.cl_last_error(engine.handle)
    # valid ids go through afterwards
    seg[2] = 0
    (maps, tmin, npe, ctr, sampled), st = sample_sites(
        engine, BOX_BGO, OP_BGO_ESR, GRID, TB80, xyz=xyz, t0=t0, photons=ph, segment=seg, n_segments=2, seed=3,
        tau_ns=1768.0, light=light)
    assert int(sampled[0]) == 4000 and int(npe.sum()) == int(sampled[1]) > 0


def test_transport_source_with_a_bad_segment_is_reported(engine):
    """cl_run_segments_device trusts its device arrays; a segment id outside
    the maps still cannot write out of range: its detections are dropped and
    the sync reports CL_ERR_ARG."""
    import torch
    from crysplight_b200 import _lib
    from crysplight_b200._lib import CudaTransportError
    dev = "cuda"
    sx = torch.tensor([24.0, 24.0], device=dev)
    sy = torch.tensor([24.0, 24.0], device=dev)
    sz = torch.tensor([20.0, 20.0], device=dev)
    off = torch.tensor([0, 500, 1000], dtype=torch.int64, device=dev)
    seg = torch.tensor([0, 5], dtype=torch.int32, device=dev)           # 5 >= n_segments
    maps = torch.zeros(64 * 2, dtype=torch.int32, device=dev)
    tmin = torch.zeros(64 * 2, dtype=torch.float32, device=dev)
    npe = torch.zeros(2, dtype=torch.int32, device=dev)
    ctr = torch.zeros(9, dtype=torch.int64, device=dev)
    st = torch.cuda.Stream()
    engine.run_segments_device(BOX_BGO, OP_BGO_ESR, GRID, TB80, sx=sx.data_ptr(), sy=sy.data_ptr(), sz=sz.data_ptr(),
                               st=None, src_offsets=off.data_ptr(), src_segment=seg.data_ptr(), n_src=2,
                               n_segments=2, n_photons=1000, seed=4, tau_ns=0.0, maps=maps.data_ptr(),
                               tmin=tmin.data_ptr(), npe=npe.data_ptr(), counters=ctr.data_ptr(),
                               stream=st.cuda_stream)
    with pytest.raises(CudaTransportError) as e:
        engine.sync(st.cuda_stream)
    assert e.value.code == _lib.CL_ERR_ARG
    assert int(maps[64:].sum()) == 0 and int(npe[0]) == int(maps[:64].sum()) > 0
