"""Drop-in check on the reference's own input files: every run file under the
reference's runs/ and every material file under its data/ is read unchanged
(comments, inline comments and all) by the Python mirror of load_setup
(src/config.jl:27-69, src/materials.jl:8-12), by the gamma-campaign loader
(scripts/shoot_gammas.jl:19-45) and by crysplight_run --print-setup, and gives
the same setup as this package's comment-free copies.  Skipped where the
reference checkout is absent."""
import glob
import json
import os
import subprocess
import tomllib

import numpy as np
import pytest

from crysplight_b200.config import PKG_DATA_DIR, PKG_RUNS_DIR, load_setup
from crysplight_b200.shoot_gammas import load_gamma_setup

REF = os.environ.get("CRYSPLIGHT_REFERENCE", "/root/reference")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "crysplight_b200", "lib", "crysplight_run")

pytestmark = pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "runs")),
                                reason="reference checkout not present")

POINT_RUNS = sorted(glob.glob(os.path.join(REF, "runs", "point_*.toml")))
GAMMA_RUNS = sorted(glob.glob(os.path.join(REF, "runs", "gammas_*.toml")))
MATERIALS = sorted(glob.glob(os.path.join(REF, "data", "*.toml")))


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-C", os.path.join(ROOT, "crysplight_b200", "csrc")], check=True,
                       capture_output=True)
    return CLI


def _cli_setup(cli, path):
    r = subprocess.run([cli, "--print-setup", path], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def _physics(st, ro_grid):
    f32 = np.float32
    op = st.op
    return ([f32(v) for v in st.box.L],
            [f32(getattr(op, k)) for k in ("n_crystal", "n_coupling", "abs_len_mm", "rayleigh_mm",
                                           "wrap_R", "sigma_alpha", "pde")],
            (op.wrap_specular, op.air_gap),
            (f32(ro_grid.pitch_mm), ro_grid.nx, ro_grid.ny),
            (f32(st.tb.bin_ns), st.tb.nbins), f32(st.tau_ns))


def test_the_reference_ships_the_files_the_runs_name():
    assert len(POINT_RUNS) >= 4 and len(GAMMA_RUNS) >= 6 and len(MATERIALS) >= 7


@pytest.mark.parametrize("path", MATERIALS, ids=os.path.basename)
def test_material_files_match_the_package_copies(path):
    """The package's data/ copies hold the same keys and values (comments stripped)."""
    mine = os.path.join(PKG_DATA_DIR, os.path.basename(path))
    if not os.path.exists(mine):
        pytest.skip(f"no package copy of {os.path.basename(path)} (no run file of this package uses it)")
    with open(path, "rb") as f:
        ref = tomllib.load(f)
    with open(mine, "rb") as f:
        cp = tomllib.load(f)
    assert ref == cp


@pytest.mark.parametrize("path", POINT_RUNS, ids=os.path.basename)
def test_point_runs_read_unchanged(cli, path):
    st = load_setup(path)
    j = _cli_setup(cli, path)
    f32 = np.float32
    assert j["tag"] == st.tag
    assert [f32(v) for v in j["box"]] == [f32(v) for v in st.box.L]
    for k in ("n_crystal", "n_coupling", "abs_len_mm", "rayleigh_mm", "wrap_R", "sigma_alpha", "pde"):
        assert f32(j["op"][k]) == f32(getattr(st.op, k)), k
    assert (j["op"]["wrap_specular"], j["op"]["air_gap"]) == (st.op.wrap_specular, st.op.air_gap)
    assert j["tb"][1] == st.tb.nbins and [f32(v) for v in j["pos"]] == [f32(v) for v in st.pos]
    assert (j["n_photons"], j["seed"], j["max_bounces"]) == (st.n_photons, st.seed, st.max_bounces)
    mine = os.path.join(PKG_RUNS_DIR, os.path.basename(path))
    if os.path.exists(mine):
        cp = load_setup(mine)
        assert _physics(st, st.grid) == _physics(cp, cp.grid)
        assert (st.tag, st.pos, st.n_photons, st.seed, st.max_bounces) == \
            (cp.tag, cp.pos, cp.n_photons, cp.seed, cp.max_bounces)


@pytest.mark.parametrize("path", GAMMA_RUNS, ids=os.path.basename)
def test_gamma_campaigns_read_unchanged(cli, path):
    st = load_gamma_setup(path)
    j = _cli_setup(cli, path)
    f32 = np.float32
    assert j["tag"] == st.tag and (j["n_events"], j["seed"]) == (st.n_events, st.seed)
    for k in ("n_crystal", "n_coupling", "abs_len_mm", "rayleigh_mm", "wrap_R", "sigma_alpha", "pde"):
        assert f32(j["op"][k]) == f32(getattr(st.op, k)), k
    assert j["tb"][1] == st.tb.nbins and j["yield_per_mev"] == st.yield_per_mev
    assert os.path.realpath(j["xcom"]) == os.path.realpath(st.xcom_path)
    assert os.path.isfile(st.xcom_path)
    mine = os.path.join(PKG_RUNS_DIR, os.path.basename(path))
    if os.path.exists(mine):
        cp = load_gamma_setup(mine)
        assert _physics(st, st.ro.grid) == _physics(cp, cp.ro.grid)
        assert (st.tag, st.n_events, st.seed, st.yield_per_mev, st.density, st.crystal_name) == \
            (cp.tag, cp.n_events, cp.seed, cp.yield_per_mev, cp.density, cp.crystal_name)
        with open(st.xcom_path, "rb") as a, open(cp.xcom_path, "rb") as b:
            assert a.read() == b.read()
