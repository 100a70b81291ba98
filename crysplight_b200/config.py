"""Run configuration: the reference's run TOMLs and material files.

Mirrors src/config.jl (``RunSetup``, ``load_setup``, ``run_from_config``) and
src/materials.jl (``load_material``).  A run file ``runs/<tag>.toml`` names
materials that live in ``data/<name>.toml``; by default the data directory is
the run file's ``../data`` (the reference's layout), falling back to this
package's copy of the standard materials.
"""
from __future__ import annotations

import os
import time
import tomllib
from dataclasses import dataclass, field
from typing import Optional

from .params import (Box, OpticalParams, SipmGrid, TimeBinning, deg2rad_f32, f32,
                     surface_has_gap)

PKG_DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
PKG_RUNS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "runs")


def load_material(name: str, data_dir: Optional[str] = None) -> dict:
    """data/<name>.toml as a dict (src/materials.jl:8-12)."""
    path = os.path.join(data_dir or PKG_DATA_DIR, name + ".toml")
    if not os.path.isfile(path):
        raise FileNotFoundError(f"material file not found: {path}")
    with open(path, "rb") as f:
        return tomllib.load(f)


def _data_dir_for(cfg_path: str) -> str:
    cand = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(cfg_path))), "data")
    return cand if os.path.isdir(cand) else PKG_DATA_DIR


def julia_round(x: float) -> int:
    """Julia's round(): nearest, ties to even (as Python's round)."""
    return int(round(x))


@dataclass
class RunSetup:
    """src/config.jl:5-19."""
    tag: str
    cfg: dict
    box: Box
    op: OpticalParams
    grid: SipmGrid
    tb: TimeBinning
    pos: tuple
    tau_ns: float
    n_photons: int
    seed: int
    max_bounces: int
    outdir: str
    cfg_path: str


def optical_from(crystal: dict, wrap: dict, sipm: dict, cfg: dict) -> OpticalParams:
    """OpticalParams as built in src/config.jl:39-50."""
    pde = f32(cfg["sipm"].get("pde_override", sipm["pde"]))
    surf = cfg.get("surface", {})
    finish = surf.get("finish", "backpainted")
    return OpticalParams(f32(crystal["n"]), f32(cfg["sipm"]["coupling_n"]),
                         f32(crystal["abs_length_mm"]),
                         f32(crystal.get("rayleigh_mm", float("inf"))),
                         f32(wrap["reflectivity"]), wrap["model"] == "specular",
                         surface_has_gap(finish),
                         deg2rad_f32(surf.get("sigma_alpha_deg", 0.0)), pde)


def time_binning_from(binning: dict) -> TimeBinning:
    bin_ns = f32(binning["bin_ns"])
    return TimeBinning(bin_ns, julia_round(binning["window_ns"] / bin_ns))


def load_setup(cfg_path: str, data_dir: Optional[str] = None) -> RunSetup:
    """load_setup, src/config.jl:27-69."""
    with open(cfg_path, "rb") as f:
        cfg = tomllib.load(f)
    data_dir = data_dir or _data_dir_for(cfg_path)
    run = cfg["run"]
    tag = run.get("tag", os.path.splitext(os.path.basename(cfg_path))[0])
    crystal = load_material(cfg["crystal"]["material"], data_dir)
    wrap = load_material(cfg["wrap"]["material"], data_dir)
    sipm = load_material(cfg["sipm"]["material"], data_dir)
    sz = [f32(v) for v in cfg["crystal"]["size_mm"]]
    box = Box((sz[0], sz[1], sz[2]))
    op = optical_from(crystal, wrap, sipm, cfg)
    grid = SipmGrid(f32(sipm["pitch_mm"]), int(sipm["nx"]), int(sipm["ny"]))
    tb = time_binning_from(cfg["binning"])
    src = cfg["source"]
    if src["type"] != "point":
        raise ValueError("v0 supports only the point source")
    p = tuple(f32(v) for v in src["position_mm"])
    tau = 0.0 if src["time_profile"] == "delta" else f32(crystal["tau_ns"])
    outdir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(cfg_path))),
                          cfg.get("output", {}).get("dir", "output"), tag)
    return RunSetup(tag, cfg, box, op, grid, tb, p, tau, int(run["n_photons"]), int(run["seed"]),
                    int(run.get("max_bounces", 100_000)), outdir, os.path.abspath(cfg_path))


def run_from_config(cfg_path: str, *, engine=None, data_dir: Optional[str] = None,
                    write: bool = True) -> dict:
    """run_from_config, src/config.jl:72-79: transport on the GPU, write output/<tag>/."""
    from .transport import default_engine
    from .output import write_output
    st = load_setup(cfg_path, data_dir)
    eng = engine or default_engine()
    t0 = time.perf_counter()
    acc = eng.run_photons(st.box, st.op, st.grid, st.tb, n_photons=st.n_photons, seed=st.seed,
                          pos=st.pos, tau_ns=st.tau_ns, max_bounces=st.max_bounces)
    elapsed = time.perf_counter() - t0
    return write_output(st, acc, elapsed, write=write)
