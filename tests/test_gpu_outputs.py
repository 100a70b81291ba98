"""The drivers end to end on the GPU: run_from_config writes light.h5 and
shoot_gammas writes events.h5 (plain Monte Carlo and surrogate with
fallback), read back with the package's HDF5 reader and checked for the
reference's invariants (scripts/shoot_gammas.jl:60-90, src/output.jl:10-32)."""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNS = os.path.join(ROOT, "crysplight_b200", "runs")


def _copy_run(tmp_path, name):
    runs = tmp_path / "runs"
    runs.mkdir(exist_ok=True)
    dst = runs / name
    shutil.copy(os.path.join(RUNS, name), dst)
    return str(dst)


def test_run_from_config_writes_light_h5(engine, tmp_path):
    from crysplight_b200.config import run_from_config
    from crysplight_b200.hdf5 import read_h5
    cfg = _copy_run(tmp_path, "point_csitl_teflon.toml")
    s = run_from_config(cfg, engine=engine)
    d, a = read_h5(str(tmp_path / "output" / "point_csitl_teflon" / "light.h5"))
    assert d["counts"].shape == (8, 8, 81) and int(d["counts"].sum()) == a["ndet"]
    assert a["n_photons"] == 1_000_000 and a["ndet"] + a["nabs_bulk"] + a["nabs_wall"] + a["nabs_sipm"] \
        + a["ncap"] + a["nabs_surround"] == a["n_photons"]
    hit = d["counts"].sum(2) > 0
    assert np.isfinite(d["first_time_ns"][hit]).all() and np.isinf(d["first_time_ns"][~hit]).all()
    assert abs(s["detected_fraction"] - 0.888) < 0.005          # latex/csitl_calib.tex:305


def _check_events(path, n):
    from crysplight_b200.hdf5 import read_h5
    d, a = read_h5(path)
    assert d["maps"].shape == (8, 8, n) and d["tmin_ns"].shape == (8, 8, n) and d["xyz1_mm"].shape == (3, n)
    assert np.array_equal(d["maps"].reshape(64, n).sum(0), d["npe"])
    hit = d["maps"] > 0
    assert np.isfinite(d["tmin_ns"][hit]).all() and np.isinf(d["tmin_ns"][~hit]).all()
    assert ((d["edep_kev"] > 0) == (d["int_type"] >= 0)).all()
    assert a["n_events"] == n and a["tmin_nohit"] == "Inf"
    return d, a


def test_shoot_gammas_writes_events_h5(engine, tmp_path):
    from crysplight_b200.shoot_gammas import shoot_gammas
    cfg = _copy_run(tmp_path, "gammas_csitl_50k.toml")
    s = shoot_gammas(cfg, engine=engine, n_events=400)
    d, a = _check_events(str(tmp_path / "output" / "gammas_csitl_50k" / "events.h5"), 400)
    assert a["backend"] == "cuda" and a["crystal"] == "csitl" and abs(a["pde"] - 0.4) < 1e-7
    peak = d["edep_kev"] > 510
    assert 5000 < d["npe"][peak].mean() < 15000                  # test/runtests.jl:330-332


def test_shoot_gammas_with_the_surrogate(engine, tmp_path):
    from crysplight_b200.fast_events import SurrogateEvents
    from crysplight_b200.shoot_gammas import shoot_gammas
    from crysplight_b200.surrogate import LightSurrogate
    cfg = _copy_run(tmp_path, "gammas_bgo_esr_500k.toml")
    se = SurrogateEvents(LightSurrogate.load(os.path.join(ROOT, "crysplight_b200", "surrogates", "bgo_esr.npz")),
                         engine)
    try:
        s = shoot_gammas(cfg, engine=engine, surrogate=se, n_events=3000)
    finally:
        se.close()
    d, a = _check_events(str(tmp_path / "output" / "gammas_bgo_esr_500k" / "events.h5"), 3000)
    assert a["backend"] == "cuda-surrogate"
    peak = d["edep_kev"] > 510
    assert abs(d["npe"][peak].mean() / 2004.0 - 1) < 0.02        # the plain Monte Carlo's photopeak
    st = s["result"].surrogate_stats
    assert 0 < st["fallback_sites"] < st["sites"]


def test_run_point_source_cli(tmp_path, capsys):
    from crysplight_b200.run_point_source import main
    cfg = _copy_run(tmp_path, "point_bgo_esr.toml")
    main([cfg])
    out = capsys.readouterr().out
    assert "detected" in out and os.path.exists(tmp_path / "output" / "point_bgo_esr" / "light.h5")
