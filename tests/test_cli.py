"""crysplight_run, the C++ host program over the C-ABI (no Python): its run-file
parsing against the Python mirror of load_setup (src/config.jl:27-69), its
HDF5 writer against crysplight_b200/hdf5.py byte for byte, and (GPU) its
light.h5 against the one run_from_config writes for the same run file."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from crysplight_b200.config import load_setup
from crysplight_b200.shoot_gammas import load_gamma_setup

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "crysplight_b200")
CLI = os.path.join(PKG, "lib", "crysplight_run")
RUNS = [os.path.join(PKG, "runs", f) for f in ("point_csitl_teflon.toml", "point_bgo_esr.toml")]
GAMMA_RUNS = [os.path.join(PKG, "runs", f) for f in ("gammas_csitl_50k.toml", "gammas_bgo_500k.toml",
                                                      "gammas_bgo_esr_500k.toml")]


@pytest.fixture(scope="module")
def cli():
    if not os.path.exists(CLI):
        subprocess.run(["make", "-C", os.path.join(PKG, "csrc")], check=True, capture_output=True)
    assert os.access(CLI, os.X_OK)
    return CLI


def _setup_json(cli, path, *extra):
    r = subprocess.run([cli, "--print-setup", *extra, path], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def _same_setup(j, st):
    f32 = np.float32
    assert j["tag"] == st.tag
    assert os.path.realpath(j["outdir"]) == os.path.realpath(st.outdir)
    assert [f32(v) for v in j["box"]] == [f32(v) for v in st.box.L]
    for k in ("n_crystal", "n_coupling", "abs_len_mm", "rayleigh_mm", "wrap_R", "sigma_alpha", "pde"):
        assert f32(j["op"][k]) == f32(getattr(st.op, k)), k
    assert j["op"]["wrap_specular"] == st.op.wrap_specular and j["op"]["air_gap"] == st.op.air_gap
    assert f32(j["grid"][0]) == f32(st.grid.pitch_mm) and j["grid"][1:] == [st.grid.nx, st.grid.ny]
    assert f32(j["tb"][0]) == f32(st.tb.bin_ns) and j["tb"][1] == st.tb.nbins
    assert [f32(v) for v in j["pos"]] == [f32(v) for v in st.pos]
    assert f32(j["tau_ns"]) == f32(st.tau_ns)
    assert (j["n_photons"], j["seed"], j["max_bounces"]) == (st.n_photons, st.seed, st.max_bounces)
    assert (j["crystal"], j["wrap"]) == (st.cfg["crystal"]["material"], st.cfg["wrap"]["material"])
    assert j["finish"] == st.cfg.get("surface", {}).get("finish", "backpainted")
    assert j["sigma_alpha_deg"] == float(st.cfg.get("surface", {}).get("sigma_alpha_deg", 0.0))


@pytest.mark.parametrize("path", RUNS)
def test_setup_matches_the_python_mirror(cli, path):
    _same_setup(_setup_json(cli, path), load_setup(path))


RUN_VARIANT = """# edge cases of the TOML subset: comments, underscores, spacing, a tag,
# a multi-line array, literal strings, an explicit max_bounces
[run]
n_photons = 1_000   # photons
seed = 0x2A
tag = "edge \\"case\\""
max_bounces = 5_000

[crystal]
material = 'bgo'
size_mm = [
    30.0,   # x
    31.5,
    1e1,
]

[wrap]
material = "teflon"

[sipm]
material = "sipm_s14160"
coupling_n = 1.5

[surface]
finish = "frontpainted"

[source]
type = "point"
position_mm = [1, 2.5, 3]
time_profile = "delta"

[binning]
bin_ns = 25.0
window_ns = 1012.5

[output]
dir = "elsewhere"
"""


@pytest.mark.parametrize("path", GAMMA_RUNS)
def test_gamma_campaign_setup_matches_the_python_mirror(cli, path):
    j = _setup_json(cli, path)
    st = load_gamma_setup(path)
    f32 = np.float32
    assert j["tag"] == st.tag and os.path.realpath(j["outdir"]) == os.path.realpath(st.outdir)
    assert [f32(v) for v in j["box"]] == [f32(v) for v in st.box.L]
    for k in ("n_crystal", "n_coupling", "abs_len_mm", "rayleigh_mm", "wrap_R", "sigma_alpha", "pde"):
        assert f32(j["op"][k]) == f32(getattr(st.op, k)), k
    assert j["op"]["wrap_specular"] == st.op.wrap_specular and j["op"]["air_gap"] == st.op.air_gap
    assert f32(j["grid"][0]) == f32(st.ro.grid.pitch_mm) and j["grid"][1:] == [st.ro.grid.nx, st.ro.grid.ny]
    assert f32(j["tb"][0]) == f32(st.tb.bin_ns) and j["tb"][1] == st.tb.nbins
    assert j["yield_per_mev"] == st.yield_per_mev and f32(j["tau_ns"]) == f32(st.tau_ns)
    assert (j["n_events"], j["seed"]) == (st.n_events, st.seed)
    assert j["crystal"] == st.cfg["crystal"]["material"] and j["density"] == st.density
    assert os.path.realpath(j["xcom"]) == os.path.realpath(st.xcom_path)
    assert _setup_json(cli, path, "--n-events", "7")["n_events"] == 7


def test_toml_subset_edge_cases(cli, tmp_path):
    runs = tmp_path / "runs"
    runs.mkdir()
    p = runs / "edge.toml"
    p.write_text(RUN_VARIANT)
    data = os.path.join(PKG, "data")
    j = _setup_json(cli, str(p), "--data", data)
    st = load_setup(str(p), data_dir=data)
    _same_setup(j, st)
    assert j["tag"] == 'edge "case"' and j["seed"] == 42 and j["tb"][1] == 40   # 40.5 rounds to even
    assert j["op"]["air_gap"] == 0 and j["tau_ns"] == 0.0 and j["op"]["pde"] == np.float32(0.5)


@pytest.mark.parametrize("bad,msg", [
    ("[run]\nn_photons = 1_\n", "underscore"),
    ("[run]\nn_photons = 12 34\n", "after a value"),
    ("[run]\nx = {a = 1}\n", "inline tables"),
    ("[run]\nx = 1\nx = 2\n", "defined twice"),
    ("[run]\ns = \"open\n", "unterminated"),
])
def test_toml_errors_name_the_line(cli, tmp_path, bad, msg):
    p = tmp_path / "bad.toml"
    p.write_text(bad)
    r = subprocess.run([cli, "--print-setup", str(p)], capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr and "bad.toml:" in r.stderr, r.stderr


@pytest.mark.parametrize("args", [["--n-photons", "12x"], ["--n-photons", "-5"], ["--device", ""],
                                  ["--bogus"], []])
def test_bad_command_lines_exit_2(cli, args):
    r = subprocess.run([cli, *args, "--print-setup", RUNS[0]] if args else [cli], capture_output=True,
                       text=True)
    assert r.returncode == 2, (args, r.stderr)


def test_n_photons_override(cli):
    assert _setup_json(cli, RUNS[0], "--n-photons", "1234")["n_photons"] == 1234


def test_missing_material_and_unknown_finish_are_errors(cli, tmp_path):
    txt = open(RUNS[0]).read()
    p = tmp_path / "m.toml"
    p.write_text(txt.replace('material = "teflon"', 'material = "nosuch"'))
    r = subprocess.run([cli, "--print-setup", "--data", os.path.join(PKG, "data"), str(p)],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "material file not found" in r.stderr
    p.write_text(txt.replace('finish = "backpainted"', 'finish = "glossy"'))
    r = subprocess.run([cli, "--print-setup", "--data", os.path.join(PKG, "data"), str(p)],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "unknown finish: glossy" in r.stderr


def test_hdf5_writer_matches_the_python_writer(tmp_path):
    from crysplight_b200.hdf5 import read_h5, write_h5
    exe = tmp_path / "h5_writer_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-o", str(exe), os.path.join(ROOT, "tests", "cpp", "h5_writer_check.cpp")],
                   check=True)
    out_c = tmp_path / "c.h5"
    subprocess.run([str(exe), str(out_c)], check=True)
    counts = (7 * np.arange(24, dtype=np.uint32) + 1).reshape((3, 2, 4), order="F")
    ff = np.float32(0.5) * np.arange(6, dtype=np.float32)
    ff[4] = np.inf
    first = ff.reshape((3, 2), order="F")
    out_p = tmp_path / "p.h5"
    i8 = np.array([-1, 0, 1, 2, -128, 127], np.int8).reshape((2, 3), order="F")
    write_h5(str(out_p), {"counts": counts, "first_time_ns": first, "empty": np.zeros(0, np.float64),
                          "int_type": i8, "n_int": np.array([-1, 2, -32768], np.int16),
                          "maps": np.array([1, 65535, 0x1234], np.uint16)},
             {"tag": "h5 check", "n_photons": np.int64(1000000), "bin_ns": np.float32(100.0),
              "nbins": np.int32(80), "flag": np.uint8(1), "big": np.uint64(0xFFFFFFFFFFFFFFF0),
              "u32": np.uint32(4000000000), "sigma_alpha_deg": np.float64(1.3), "empty_str": ""})
    assert out_c.read_bytes() == out_p.read_bytes()
    d, a = read_h5(str(out_c))
    assert np.array_equal(d["counts"], counts) and a["tag"] == "h5 check"
    assert np.array_equal(d["first_time_ns"], first)


@pytest.mark.gpu
def test_cli_gamma_campaign_writes_the_same_events_h5_as_python(cli, tmp_path):
    """A gamma campaign through crysplight_run and through shoot_gammas: the
    two events.h5 files are identical byte for byte."""
    from crysplight_b200.shoot_gammas import shoot_gammas
    from crysplight_b200.transport import Engine
    runs = tmp_path / "runs"
    runs.mkdir()
    for src in GAMMA_RUNS[:2]:
        p = runs / os.path.basename(src)
        p.write_text(open(src).read())
        eng = Engine(0)
        try:
            shoot_gammas(str(p), engine=eng, n_events=400)
        finally:
            eng.close()
        tag = load_gamma_setup(str(p)).tag
        py_file = tmp_path / "output" / tag / "events.h5"
        shutil.move(str(py_file), str(tmp_path / f"{tag}.py.h5"))
        r = subprocess.run([cli, "--n-events", "400", str(p)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert "events" in r.stdout and "interacted" in r.stdout
        assert (tmp_path / f"{tag}.py.h5").read_bytes() == py_file.read_bytes()


@pytest.mark.gpu
def test_cli_run_writes_the_same_light_h5_as_python(cli, tmp_path):
    """Same run file through crysplight_run and through run_from_config: the
    two light.h5 files are identical byte for byte."""
    from crysplight_b200.config import run_from_config
    from crysplight_b200.transport import Engine
    runs = tmp_path / "runs"
    runs.mkdir()
    for src in RUNS:
        txt = open(src).read().replace("n_photons = 1000000", "n_photons = 300000")
        p = runs / os.path.basename(src)
        p.write_text(txt)
        eng = Engine(0)
        try:
            run_from_config(str(p), engine=eng)
        finally:
            eng.close()
        tag = os.path.splitext(os.path.basename(src))[0]
        py_file = tmp_path / "output" / tag / "light.h5"
        shutil.move(str(py_file), str(tmp_path / f"{tag}.py.h5"))
        r = subprocess.run([cli, str(p)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert "detected" in r.stdout
        assert (tmp_path / f"{tag}.py.h5").read_bytes() == py_file.read_bytes()


def test_campaign_without_events_is_an_error(cli, tmp_path):
    """campaign.n_events < 1 (in the run file or from --n-events) is rejected
    with a message, by the C++ program and by the Python loader."""
    runs = tmp_path / "runs"
    runs.mkdir()
    txt = open(GAMMA_RUNS[0]).read()
    import re
    p = runs / "zero.toml"
    p.write_text(re.sub(r"n_events\s*=\s*[0-9_]+", "n_events = 0", txt))
    r = subprocess.run([cli, "--print-setup", "--data", os.path.join(PKG, "data"), str(p)],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "n_events must be >= 1" in r.stderr
    with pytest.raises(ValueError):
        load_gamma_setup(str(p), data_dir=os.path.join(PKG, "data"))
    r = subprocess.run([cli, "--print-setup", "--n-events", "0", GAMMA_RUNS[0]], capture_output=True, text=True)
    assert r.returncode != 0 and "n-events" in r.stderr


def test_summary_with_one_photopeak_event(capsys):
    """The reference prints the photopeak line whenever a photopeak event
    exists (scripts/shoot_gammas.jl:86-89); with one event the width is NaN."""
    from types import SimpleNamespace
    from crysplight_b200.shoot_gammas import summary
    st = load_gamma_setup(GAMMA_RUNS[0])
    st.n_events = 3
    r = SimpleNamespace(edep=np.float32([511.0, 0.0, 300.0]), npe=np.int32([9800, 0, 5000]))
    out = summary(st, r, 1.0, "cuda")
    line = capsys.readouterr().out.splitlines()[-1]
    assert "9800 pe mean" in line and "NaN%" in line and out["photopeak_pe_mean"] == 9800.0
