"""Host-side pieces of the surrogate: persistence, input scaling, the grid,
the held-out baselines and the event-comparison statistics.  No GPU."""
import numpy as np
import pytest

from crysplight_b200.params import Box
from crysplight_b200.surrogate import (LightSurrogate, depth_unwarp, depth_warp, grid_points, light_targets,
                                       split_holdout, ScanResult)


def test_save_load_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    s = LightSurrogate(np.array([48.0, 48.0, 22.4]), rng.standard_normal(192).astype(np.float32),
                       np.abs(rng.standard_normal(192)).astype(np.float32) + 0.1,
                       [rng.standard_normal(10).astype(np.float32) for _ in range(3)], z_warp=0.25)
    p = str(tmp_path / "m.npz")
    s.save(p)
    t = LightSurrogate.load(p)
    assert np.array_equal(t.box_mm, s.box_mm) and np.array_equal(t.y_mean, s.y_mean)
    assert np.array_equal(t.y_std, s.y_std) and len(t.members) == 3 and t.z_warp == 0.25
    assert all(np.array_equal(a, b) for a, b in zip(t.members, s.members))


def test_inputs_and_depth_warp():
    s = LightSurrogate(np.array([48.0, 48.0, 22.4]), np.zeros(192), np.ones(192), [])
    x = s.normalise([[0.0, 24.0, 22.4], [48.0, 12.0, 0.0]])
    assert np.allclose(x, [[-1, 0, 1], [1, -0.5, -1]])
    w = np.linspace(0, 1, 101)
    for a in (0.0, 0.3, 0.9):
        t = depth_unwarp(w, a)
        assert np.allclose(depth_warp(t, a), w, atol=1e-12)
        assert np.all(np.diff(depth_warp(np.linspace(0, 1, 50), a)) > 0)
    s.z_warp = 0.5
    z = s.normalise([[1.0, 1.0, 11.2]])[0, 2]
    assert z == pytest.approx(2 * depth_warp(0.5, 0.5) - 1, abs=1e-6)


def test_depth_slab_inputs_grid_and_persistence(tmp_path):
    """An expert for the slab z0..z1: its grid lies in the slab, its network
    input maps the slab onto [-1, 1] (clamped outside), and the range survives
    save/load (the whole-crystal ensembles keep z_range None)."""
    box = Box((48.0, 48.0, 22.4))
    g = grid_points(box, (2, 2, 4), z_range=(14.4, 22.4))
    assert np.allclose(np.unique(g[:, 2]), [15.4, 17.4, 19.4, 21.4])
    s = LightSurrogate(np.array([48.0, 48.0, 22.4]), np.zeros(192), np.ones(192),
                       [np.zeros(4, np.float32)], z_range=(14.4, 22.4))
    assert s.depth_range() == (14.4, 22.4)
    x = s.normalise([[0.0, 48.0, 14.4], [24.0, 24.0, 22.4], [24.0, 24.0, 18.4], [1.0, 1.0, 3.0]])
    assert np.allclose(x[:, 2], [-1.0, 1.0, 0.0, -1.0], atol=1e-6)
    assert np.allclose(x[:, :2], [[-1, 1], [0, 0], [0, 0], [2 / 48 - 1, 2 / 48 - 1]])
    p = str(tmp_path / "slab.npz")
    s.save(p)
    assert LightSurrogate.load(p).z_range == (14.4, 22.4)
    w = LightSurrogate(np.array([48.0, 48.0, 22.4]), np.zeros(192), np.ones(192), [np.zeros(4, np.float32)])
    w.save(p)
    t = LightSurrogate.load(p)
    assert t.z_range is None and t.depth_range() == (0.0, 22.4)


def test_grid_and_holdout():
    box = Box((48.0, 48.0, 22.4))
    g = grid_points(box, (4, 3, 2))
    assert g.shape == (24, 3) and np.allclose(g[:4, 0], [6, 18, 30, 42]) and np.allclose(g[0], [6, 8, 5.6])
    gw = grid_points(box, (1, 1, 24), z_warp=0.5)
    assert np.all(np.diff(gw[:, 2]) > 0) and gw[-1, 2] < 22.4 and np.diff(gw[:, 2])[-1] < np.diff(gw[:, 2])[0]
    tr, ho = split_holdout(1000, 0.1, seed=3)
    assert ho.size == 100 and tr.size == 900 and not np.intersect1d(tr, ho).size


def test_targets_from_counts_and_moments():
    from crysplight_b200 import _lib
    counts = np.array([[1000, 10, 0, 5000]], np.int64)
    t = np.array([[2.0, 3.0, 0.0, 1.5]])
    sig = np.array([[0.5, 0.4, 0.0, 0.2]])
    tsum = np.rint(counts * t * _lib.MOMENT_T_SCALE).astype(np.uint64)
    tsum2 = np.rint(counts * (t * t + sig * sig) * _lib.MOMENT_T2_SCALE).astype(np.uint64)
    scan = ScanResult(np.zeros((1, 3), np.float32), 100_000, counts, tsum, tsum2, np.zeros((1, 4), np.float32))
    y = light_targets(scan)
    c = 4
    assert np.allclose(np.exp(y[0, :c]), (counts[0] + 0.5) / 100_001)
    assert y[0, c] == pytest.approx(2.0, abs=1e-5) and y[0, c + 3] == pytest.approx(1.5, abs=1e-5)
    assert y[0, 2 * c] == pytest.approx(np.log(0.5), abs=1e-4)


def test_table_baseline_and_error_metric():
    from crysplight_b200.surrogate_train import rel_error, table_interpolate
    box = Box((48.0, 48.0, 22.4))
    shape = (6, 5, 4)
    pts = grid_points(box, shape)
    vals = np.stack([pts[:, 0] * 2 + pts[:, 1] - pts[:, 2] + 100, pts[:, 2] + 10], 1).astype(np.float64)
    inner = np.array([1 + 6 * (1 + 5 * 1), 2 + 6 * (2 + 5 * 2)])      # interior nodes
    tr = np.setdiff1d(np.arange(pts.shape[0]), inner)
    out = table_interpolate(shape, tr, vals, inner)
    assert np.allclose(out, vals[inner])                              # linear fields: exact midpoints
    e = rel_error(np.array([[1.02, 0.5]]), np.array([[1.0, 0.4]]), 1000)
    assert e["cells"] == 2 and e["mean"] == pytest.approx((0.02 + 0.25) / 2)


def test_photopeak_and_map_comparison():
    from crysplight_b200.fast_events import compare_maps, photopeak
    rng = np.random.default_rng(1)
    edep = np.where(rng.uniform(size=20000) < 0.6, 511.0, rng.uniform(0, 500, 20000))
    npe = rng.normal(2000, 45, 20000)
    pk = photopeak(npe, edep)
    assert pk["events"] == int((edep == 511).sum()) and abs(pk["mean"] - 2000) < 3 and abs(pk["sigma"] - 45) < 2
    lam = rng.uniform(5, 50, size=(8, 8, 1))
    a = rng.poisson(lam, size=(8, 8, 5000))
    b = rng.poisson(lam, size=(8, 8, 5000))
    cmp = compare_maps(a, b)
    assert 0.95 < cmp["chi2_ndf_mean"] < 1.05 and cmp["rel_mean"] < 0.01
