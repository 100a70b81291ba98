"""The shipped light-response ensembles against a fresh high-statistics Monte
Carlo at held-out grid nodes: the acceptance bar of the surrogate is a mean
per-SiPM relative error of the detection probabilities (the per-SiPM counts
of src/transport.jl:96-108 divided by the photons emitted) of at most 1%.

The held-out nodes are the ones the ensembles never saw: the 48x48x24 grid of
cell centres the training scanned, split by split_holdout(n, 0.1, seed=11) as
in surrogate_train.py.  The truth is an independent Monte Carlo (its own
seed) of 10^7 photons per node; the error is averaged over the cells whose
expected count at the training scan's 10^5 photons exceeds 100."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SURROGATES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                          "crysplight_b200", "surrogates")
TRUTH_PHOTONS = 10_000_000
TRAIN_PHOTONS = 100_000


def _holdout(engine, setup_name: str, model: str, n_nodes: int, seed: int):
    from crysplight_b200.surrogate import LightSurrogate, grid_points, scan_light, split_holdout
    from crysplight_b200.surrogate_train import rel_error, setup
    box, op, ro = setup(setup_name)
    sur = LightSurrogate.load(os.path.join(SURROGATES, model))
    pts = grid_points(box, (48, 48, 24))
    tr, ho = split_holdout(pts.shape[0], 0.1, seed=11)
    assert np.intersect1d(tr, ho).size == 0
    rng = np.random.default_rng(5)
    sub = np.sort(rng.choice(ho, size=n_nodes, replace=False))
    truth = scan_light(engine, box, op, ro, points=pts[sub], photons_per_point=TRUTH_PHOTONS, seed=seed,
                       batch_points=64)
    p_true = truth.counts / float(TRUTH_PHOTONS)
    pred = sur.predict(pts[sub])
    q = pts[sub].astype(np.float64)
    L = [float(box.L[i]) for i in range(3)]
    d_wall = np.minimum.reduce([q[:, 0], L[0] - q[:, 0], q[:, 1], L[1] - q[:, 1], q[:, 2]])
    served = (d_wall >= 1.0) & (pred["spread"] <= 0.02)
    return (rel_error(pred["p"], p_true, TRAIN_PHOTONS),
            rel_error(pred["p"][served], p_true[served], TRAIN_PHOTONS), int(served.sum()))


def test_csitl_teflon_ensemble_is_within_one_percent(engine):
    """Config 4: the CsI(Tl)+Teflon ensemble meets the 1% bar on all held-out nodes."""
    err, served, n_served = _holdout(engine, "csitl_teflon", "csitl_teflon.npz", 128, seed=90_001)
    print(f"csitl_teflon held-out error: all {err['mean']:.4f} ({err['cells']} cells), "
          f"served {served['mean']:.4f} ({n_served} nodes)")
    assert err["cells"] > 1000
    assert err["mean"] <= 0.01, err


def test_bgo_esr_ensemble_is_within_one_percent(engine):
    """Config 5's whole-crystal BGO+ESR ensemble (trained on the light minus
    its first-pass term, which it adds back exactly) meets the 1% bar on all
    held-out nodes, and on the nodes the event generator takes from it (at
    least 1 mm from a wrapped face, member spread at most 2%)."""
    err, served, n_served = _holdout(engine, "bgo_esr", "bgo_esr.npz", 128, seed=90_002)
    print(f"bgo_esr held-out error: all {err['mean']:.4f} ({err['cells']} cells), "
          f"served {served['mean']:.4f} ({n_served} nodes)")
    assert err["cells"] > 1000
    assert err["mean"] <= 0.01, err
    assert n_served >= 100
    assert served["mean"] <= 0.01, served


def test_bgo_esr_readout_face_expert_is_within_one_percent(engine):
    """The readout-face expert (64x64x16 nodes over the last 8 mm, where a
    site's light concentrates under one SiPM) on its own held-out nodes: within
    1%, and its members agree to 2% on nearly all of them, so the spread rule
    sends few sites near the readout face to the Monte Carlo."""
    from crysplight_b200.surrogate import LightSurrogate, grid_points, scan_light, split_holdout
    from crysplight_b200.surrogate_train import rel_error, setup
    box, op, ro = setup("bgo_esr")
    sur = LightSurrogate.load(os.path.join(SURROGATES, "bgo_esr_face.npz"))
    pts = grid_points(box, (64, 64, 16), z_range=sur.z_range)
    _, ho = split_holdout(pts.shape[0], 0.1, seed=11)
    sub = np.sort(np.random.default_rng(5).choice(ho, size=96, replace=False))
    truth = scan_light(engine, box, op, ro, points=pts[sub], photons_per_point=TRUTH_PHOTONS, seed=90_003,
                       batch_points=64)
    pred = sur.predict(pts[sub])
    err = rel_error(pred["p"], truth.counts / float(TRUTH_PHOTONS), TRAIN_PHOTONS)
    flagged = float(np.mean(pred["spread"] > 0.02))
    print(f"bgo_esr_face held-out error {err['mean']:.4f} ({err['cells']} cells), spread > 2%: {flagged:.3f}")
    assert err["mean"] <= 0.01, err
    assert flagged <= 0.05
