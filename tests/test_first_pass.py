"""The surrogate's first-pass term (cl_surrogate_direct) on the CPU: its NumPy
restatement (oracle/first_pass.py) against brute-force sampling of the same
integral, and against the reference transport itself: the photons the C
restatement of run_photons_ka! (src/kernel.jl:159-367) detects with no wall
interaction and no scatter before the readout face (bounces == 0) are exactly
the first-pass photons.  The GPU kernel is checked against the restatement in
tests/test_gpu_first_pass.py."""
import numpy as np
import pytest

from crysplight_b200.params import STATUS_DETECTED, TimeBinning
from crysplight_b200.surrogate_train import setup
from oracle import first_pass as FP

BOX, OP, RO = setup("bgo_esr")
L = [float(BOX.L[i]) for i in range(3)]
ARGS = (L, float(OP.n_crystal), float(OP.n_coupling), float(OP.abs_len_mm), float(OP.rayleigh_mm), 6.0, 8, 8)


@pytest.mark.parametrize("site", [(24.0, 24.0, 21.4), (5.7, 12.3, 21.9), (30.2, 17.9, 18.0),
                                  (6.0, 6.0, 14.4), (1.5, 46.0, 22.0)])
def test_quadrature_matches_sampling(site):
    d = FP.direct([site], *ARGS)[0]
    s = FP.sample(site, *ARGS, n=2_000_000, seed=7)
    tol = 5.0 * np.sqrt(np.maximum(s, 1e-6) / 2_000_000) + 1e-6
    assert np.all(np.abs(d - s) <= tol), (d - s)[np.abs(d - s) > tol]
    assert abs(d.sum() - s.sum()) < 5.0 * np.sqrt(s.sum() / 2_000_000)


def test_quadrature_edge_cases():
    # outside the crystal, on or beyond the readout face: no first-pass light
    d = FP.direct([(24.0, 24.0, 22.4), (24.0, 24.0, 23.0), (-1.0, 5.0, 20.0)], *ARGS)
    assert np.all(d == 0.0)
    # a centred site: four-fold symmetry; every cell's probability is in [0, 1/2)
    d = FP.direct([(24.0, 24.0, 20.0)], *ARGS)[0].reshape(8, 8)
    assert np.allclose(d, d.T, rtol=1e-12) and np.allclose(d, d[::-1, ::-1], rtol=1e-12)
    assert d.max() < 0.5 and d.min() >= 0.0


@pytest.mark.parametrize("site", [(24.3, 23.1, 21.7), (9.2, 35.5, 19.9)])
def test_first_pass_is_the_reference_transports_unscattered_detections(oracle, site):
    n = 300_000
    acc, rec = oracle.run_photons_ka(BOX, OP, RO, TimeBinning(100.0, 10), n_photons=n, seed=2025,
                                     pos=site, tau_ns=0.0, return_records=True)
    first = (rec.status == STATUS_DETECTED) & (rec.bounces == 0)
    counts = np.bincount(np.abs(rec.idx[first]).astype(np.int64) - 1, minlength=64)[:64]
    d = FP.direct([site], *ARGS)[0] * n
    tol = 5.0 * np.sqrt(np.maximum(d, 1.0)) + 1.0
    assert np.all(np.abs(counts - d) <= tol), np.nonzero(np.abs(counts - d) > tol)
    assert abs(counts.sum() - d.sum()) <= 5.0 * np.sqrt(d.sum())


def test_surrogate_keeps_its_first_pass_optics(tmp_path):
    from crysplight_b200.surrogate import LightSurrogate, first_pass_optics
    from crysplight_b200.params import OpticalParams, Readout, SipmGrid
    rng = np.random.default_rng(0)
    op = OpticalParams(1.82, 1.0, float("inf"), 346.0, 1.0, True, True, 0.0, 1.0)
    fp = first_pass_optics(op, Readout(SipmGrid(6.0, 8, 8)))
    assert fp == (np.float32(1.82), 1.0, float("inf"), 346.0, 6.0, 8, 8)
    for f in (fp, None):
        s = LightSurrogate(np.array([48.0, 48.0, 22.4]), rng.standard_normal(192).astype(np.float32),
                           np.ones(192, np.float32), [rng.standard_normal(10).astype(np.float32)],
                           z_range=(14.4, 22.4), first_pass=f)
        p = str(tmp_path / "m.npz")
        s.save(p)
        t = LightSurrogate.load(p)
        assert t.first_pass == f and t.z_range == (14.4, 22.4)


def test_event_generator_refuses_other_optics():
    from types import SimpleNamespace
    from crysplight_b200.fast_events import SurrogateEvents
    from crysplight_b200.surrogate import first_pass_optics
    from crysplight_b200.params import OpticalParams
    se = SurrogateEvents.__new__(SurrogateEvents)       # the check alone, no networks on a GPU
    se.main = SimpleNamespace(sur=SimpleNamespace(first_pass=first_pass_optics(OP, RO)))
    se.experts = []
    se._check_first_pass(OP, RO)                          # the optics it was trained for
    other = OpticalParams(2.15, 1.50, 20000.0, 2222.0, 0.985, True, True, 0.0227, 0.4)
    with pytest.raises(ValueError, match="first-pass"):
        se._check_first_pass(other, RO)
    se.main = SimpleNamespace(sur=SimpleNamespace(first_pass=None))   # whole-response ensembles: any optics
    se._check_first_pass(other, RO)
