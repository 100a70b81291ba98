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


def test_max_bounces_above_the_limit_is_rejected(engine):
    """max_bounces above CL_MAX_BOUNCES_LIMIT is an argument error at every
    transport entry point (nothing is launched); <= 0 caps every photon at its
    first interaction, as src/transport.jl:228-232 does."""
    from crysplight_b200 import _lib
    from crysplight_b200._lib import CudaTransportError
    from crysplight_b200.params import Counters, Readout
    big = _lib.MAX_BOUNCES_LIMIT + 1
    with pytest.raises(CudaTransportError) as e:
        engine.run_photons_ka(BOX_BGO, OP_BGO_ESR, GRID, TB80, n_photons=100, seed=1,
                              pos=(24.0, 24.0, 11.2), tau_ns=0.0, max_bounces=big)
    assert e.value.code == _lib.CL_ERR_ARG and b"max_bounces" in engine.lib.cl_last_error(engine.handle)
    with pytest.raises(CudaTransportError) as e:
        engine.run_segments(BOX_BGO, OP_BGO_ESR, GRID, TB80, sources=[(24.0, 24.0, 11.2)],
                            photons_per_source=[100], segment_of_source=[0], n_segments=1, seed=1,
                            tau_ns=0.0, max_bounces=big)
    assert e.value.code == _lib.CL_ERR_ARG
    lib = _lib.load()
    p = np.float32([24.0])
    z = np.float32([11.2])
    counts = np.zeros(64 * 81, np.uint32)
    first = np.zeros(64, np.float32)
    ctr = Counters()
    f = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = lib.cl_run_photons_noalloc(C.byref(BOX_BGO), C.byref(OP_BGO_ESR), C.byref(Readout(GRID)),
                                    C.byref(TB80), f(p), f(p), f(z), None, 1, 100, 1, 0, 0.0, big,
                                    f(counts), f(first), C.byref(ctr), None)
    assert rc == _lib.CL_ERR_ARG and b"max_bounces" in lib.cl_last_error(None)
    # at the limit and at 0 the calls run; 0 caps each photon at its first bounce
    acc = engine.run_photons_ka(BOX_BGO, OP_BGO_ESR, GRID, TB80, n_photons=1000, seed=1,
                                pos=(24.0, 24.0, 11.2), tau_ns=0.0, max_bounces=0)
    assert acc.total_terminated() == 1000 and acc.ncap > 0


def test_time_budget_stops_a_launch_of_trapped_photons(engine):
    """Photons trapped by total internal reflection in an ideal specular box
    (src/transport.jl:228-232 bounds them by max_bounces only) keep a launch
    busy; the device time budget ends it with CL_ERR_TIMEOUT in about the
    budget's time and the handle stays usable.  Bounded without the budget
    too: 2048 photons (one per lane) x 2,000,000 bounces."""
    import time
    from crysplight_b200 import _lib
    from crysplight_b200._lib import CudaTransportError
    from cases import BOX_CSI, CENTRE_CSI, ideal
    trap = ideal(1.95, spec=True)              # wrap R = 1, no absorption, polished
    assert engine.lib.cl_set_time_budget(engine.handle, -1.0) == _lib.CL_ERR_ARG
    assert engine.lib.cl_set_time_budget(engine.handle, float("nan")) == _lib.CL_ERR_ARG
    engine.set_time_budget(0.02)
    try:
        t0 = time.perf_counter()
        with pytest.raises(CudaTransportError) as e:
            engine.run_photons_ka(BOX_CSI, trap, GRID, TB80, n_photons=2048, seed=5, pos=CENTRE_CSI,
                                  tau_ns=0.0, max_bounces=2_000_000)
        dt = time.perf_counter() - t0
        assert e.value.code == _lib.CL_ERR_TIMEOUT
        assert b"time budget" in engine.lib.cl_last_error(engine.handle)
        assert dt < 2.0, dt
    finally:
        engine.set_time_budget(_lib.DEFAULT_TIME_BUDGET_S)
    # the same photons with the reference's default cap run to completion
    acc = engine.run_photons_ka(BOX_CSI, trap, GRID, TB80, n_photons=2048, seed=5, pos=CENTRE_CSI,
                                tau_ns=0.0, max_bounces=20_000)
    assert acc.total_terminated() == 2048 and acc.ncap > 0
