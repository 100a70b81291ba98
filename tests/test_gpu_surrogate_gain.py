"""What the learned surrogate gains over the methods without it.

1. Accuracy at equal Monte Carlo budget: a small ensemble trained by the
   library's tcgen05 kernels on a coarse point scan predicts the light maps of
   held-out grid nodes better than the scan table itself (the held-out node
   interpolated from its neighbouring nodes) and better than a fresh Monte
   Carlo run of the same photon count at that node.
2. Speed at equal accuracy: the shipped BGO + ESR ensemble with Monte Carlo
   fallback generates 511 keV events faster than the plain CUDA Monte Carlo
   of the same events, with the summed-light photopeak within 0.5% and the
   per-SiPM summed light within 1%."""
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_network_beats_the_table_at_equal_budget(engine):
    from crysplight_b200.surrogate import LightSurrogate, grid_points, light_targets, scan_light, split_holdout
    from crysplight_b200.surrogate_train import rel_error, setup, table_interpolate
    box, op, ro = setup("bgo_esr")
    shape, photons = (16, 16, 8), 20_000
    pts = grid_points(box, shape)
    scan = scan_light(engine, box, op, ro, points=pts, photons_per_point=photons, seed=31)
    y = light_targets(scan)
    tr, ho = split_holdout(pts.shape[0], 0.1, seed=3)
    sub = ho[:48]
    sur = LightSurrogate.train(box, pts[tr], y[tr], members=2, steps=1500, batch=8192, lr=1e-3,
                               lr_final=1e-5, time_weight=0.1, seed=5)
    truth = scan_light(engine, box, op, ro, points=pts[sub], photons_per_point=2_000_000, seed=32,
                       batch_points=16)
    fresh = scan_light(engine, box, op, ro, points=pts[sub], photons_per_point=photons, seed=33)
    p_true = truth.counts / 2e6
    err_net = rel_error(sur.predict(pts[sub])["p"], p_true, photons)
    err_tab = rel_error(table_interpolate(shape, tr, scan.counts / photons, sub), p_true, photons)
    err_mc = rel_error(fresh.counts / photons, p_true, photons)
    print("network", err_net, "table", err_tab, "fresh MC", err_mc)
    assert err_net["mean"] < err_tab["mean"]
    assert err_net["mean"] < err_mc["mean"]


def test_fast_events_beat_the_monte_carlo(engine):
    import torch
    from bench import surrogate_events_workload
    from crysplight_b200.events import gamma_stage
    from crysplight_b200.fast_events import SurrogateEvents, compare_maps, photopeak
    from crysplight_b200.surrogate import LightSurrogate
    path = os.path.join(ROOT, "crysplight_b200", "surrogates", "bgo_esr.npz")
    E = surrogate_events_workload(20_000)
    se = SurrogateEvents(LightSurrogate.load(path), engine)
    g = gamma_stage(E["mat"], E["box"], n_events=E["n_events"], seed=E["seed"], yield_per_mev=E["yield_"])
    kw = dict(n_events=E["n_events"], seed=E["seed"], tau_ns=E["tau"], gamma=g)
    se.run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"], **kw)      # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fast = se.run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"], **kw)
    t_fast = time.perf_counter() - t0
    t0 = time.perf_counter()
    mc = engine.run_segments(E["box"], E["op"], E["ro"], E["tb"], sources=g.dep_xyz,
                             photons_per_source=g.dep_photons, segment_of_source=g.dep_event,
                             n_segments=E["n_events"], seed=E["seed"] + 1, t0s=g.dep_t, tau_ns=E["tau"])
    t_mc = time.perf_counter() - t0
    se.close()
    pk_f, pk_m = photopeak(fast.npe, g.edep), photopeak(mc.npe, g.edep)
    shift = abs(pk_f["mean"] - pk_m["mean"]) / pk_m["mean"]
    cmp = compare_maps(fast.maps.astype(np.int64), mc.maps.astype(np.int64))
    print("fast", t_fast, "mc", t_mc, fast.surrogate_stats, pk_f, pk_m, cmp)
    assert fast.surrogate_stats["fallback_sites"] < fast.surrogate_stats["sites"]
    assert t_fast < t_mc
    assert shift < 0.005
    assert abs(pk_f["fwhm_rel"] / pk_m["fwhm_rel"] - 1) < 0.1
    assert cmp["rel_mean"] < 0.01
    assert 0.8 < cmp["chi2_ndf_mean"] < 1.2
