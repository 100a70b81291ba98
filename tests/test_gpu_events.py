"""The 511 keV event pipeline on the GPU: the reference's own mini-run checks
(test/runtests.jl:305-338), bit-exactness of the optical stage given the
deposits, and the published photopeak signal of the 50k-event runs
(analysis/results/true_info/gammas_*_50k_stats.txt: npe_mean_contained)."""
import os

import numpy as np
import pytest

from crysplight_b200.events import GammaMaterial, gamma_stage, run_events
from crysplight_b200.params import Box, OpticalParams, Readout, SipmGrid, TimeBinning, deg2rad_f32

pytestmark = pytest.mark.gpu
NT = os.cpu_count() or 1
GRID = SipmGrid(6.0, 8, 8)
L_CSI = Box((48.0, 48.0, 37.2))
L_BGO = Box((48.0, 48.0, 22.4))
# runs/gammas_csitl_50k.toml: CsI(Tl) + Teflon, sigma_alpha 1.3 deg, PDE 0.40, window 8000 ns
OP_CSITL = OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, deg2rad_f32(1.3), 0.40)
# runs/gammas_bgo_50k.toml: BGO + Teflon, PDE 0.40, window 12000 ns
OP_BGO_TEF = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.99, False, True, deg2rad_f32(1.3), 0.40)


@pytest.fixture(scope="module")
def csi():
    return GammaMaterial.from_csv("CsI", 4.51, "xcom_CSI.csv")


@pytest.fixture(scope="module")
def bgo():
    return GammaMaterial.from_csv("BGO", 7.13, "xcom_BGO.csv")


def test_events_mini_run(engine, csi):               # test/runtests.jl:305-338
    r = run_events(L_CSI, OP_CSITL, Readout(GRID), TimeBinning(100.0, 80), csi, 54_000,
                   n_events=40, seed=3, tau_ns=1000.0, engine=engine)
    assert r.edep.shape == (40,) and r.maps.shape == (8, 8, 40)
    for ev in range(40):
        assert int(r.maps[:, :, ev].sum()) == r.npe[ev]
        assert (r.edep[ev] == 0) == (r.npe[ev] == 0)
        if r.edep[ev] > 510:
            assert 5000 < r.npe[ev] < 15000
        assert r.e1[ev] + r.e2[ev] + r.er[ev] == pytest.approx(511.0, abs=0.01)
        assert (r.int_type[ev] == -1) == (r.edep[ev] == 0)
        hit = r.maps[:, :, ev] > 0
        assert np.array_equal(np.isfinite(r.tmin[:, :, ev]), hit)
        assert np.all(r.tmin[:, :, ev][hit] > 0)


def test_optical_stage_matches_oracle(engine, oracle, csi):
    """Given the deposits, the batched GPU transport equals the oracle's
    per-event reduction (src/events.jl:73-87) bit for bit."""
    g = gamma_stage(csi, L_CSI, n_events=12, seed=21, yield_per_mev=54_000)
    kw = dict(sources=g.dep_xyz, photons_per_source=g.dep_photons, segment_of_source=g.dep_event,
              n_segments=12, seed=21, t0s=g.dep_t, pid_offset=0, tau_ns=1000.0)
    tb = TimeBinning(100.0, 80)
    d = engine.run_segments(L_CSI, OP_CSITL, GRID, tb, **kw)
    o = oracle.run_segments(L_CSI, OP_CSITL, GRID, tb, nthreads=NT, **kw)
    assert np.array_equal(d.maps, o["maps"])
    assert np.array_equal(d.tmin.view(np.uint32), o["tmin"].view(np.uint32))
    assert np.array_equal(d.npe, o["npe"])
    assert d.counters == o["counters"]


def test_batching_does_not_change_results(engine, csi):
    kw = dict(n_events=30, seed=5, tau_ns=1000.0, engine=engine)
    a = run_events(L_CSI, OP_CSITL, GRID, TimeBinning(100.0, 80), csi, 54_000, **kw)
    b = run_events(L_CSI, OP_CSITL, GRID, TimeBinning(100.0, 80), csi, 54_000, batch_events=7, **kw)
    assert np.array_equal(a.maps, b.maps) and np.array_equal(a.npe, b.npe)
    assert np.array_equal(a.tmin.view(np.uint32), b.tmin.view(np.uint32))


@pytest.mark.parametrize("name,box,op,yield_,tau,window,published", [
    ("csitl", L_CSI, OP_CSITL, 54_000, 1000.0, 8000.0, 9799.3),
    ("bgo", L_BGO, OP_BGO_TEF, 14_000, 1768.0, 12000.0, 2518.0),
])
def test_photopeak_signal(engine, csi, bgo, name, box, op, yield_, tau, window, published):
    """Mean photoelectrons of fully contained events (edep > 510.5 keV) within
    0.5% of the reference's published 50k-event value."""
    mat = csi if name == "csitl" else bgo
    tb = TimeBinning(100.0, int(round(window / 100.0)))
    r = run_events(box, op, GRID, tb, mat, yield_, n_events=4000, seed=11, tau_ns=tau,
                   engine=engine)
    cont = r.edep > 510.5
    mean = float(r.npe[cont].mean())
    print(name, "contained", int(cont.sum()), "npe mean", mean, "published", published)
    assert abs(mean / published - 1) < 0.005
