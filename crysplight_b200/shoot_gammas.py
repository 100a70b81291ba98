"""511 keV gamma campaigns from run files: ``scripts/shoot_gammas.jl`` on the GPU.

    python -m crysplight_b200.shoot_gammas runs/gammas_csitl_50k.toml [more.toml ...]
    python -m crysplight_b200.shoot_gammas --surrogate bgo_esr.npz runs/gammas_bgo_esr_500k.toml

For each run file: the setup is read as the reference reads it
(scripts/shoot_gammas.jl:19-45: crystal, wrap and SiPM materials from the data
directory, ``pde_override``, time binning from ``window_ns / bin_ns``, the
gamma material from ``[gamma] density`` and the XCOM table), every event runs
through ``run_events`` (all photons transported on the GPU) or, with
``--surrogate``, through the surrogate with Monte Carlo fallback, and
``output/<tag>/events.h5`` is written with the reference's datasets and root
attributes (scripts/shoot_gammas.jl:60-78), next to a copy of the run file.
The printed summary is the reference's (scripts/shoot_gammas.jl:80-90).
"""
from __future__ import annotations

import argparse
import os
import shutil
import time
import tomllib
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .config import _data_dir_for, load_material, time_binning_from
from .params import Box, OpticalParams, Readout, SipmGrid, TimeBinning, deg2rad_f32, f32, surface_has_gap

INT_TYPE_KEY = "-1 = no interaction, 0 = direct photoelectric, X>=1 = X Compton scatters"


@dataclass
class GammaSetup:
    tag: str
    cfg: dict
    cfg_path: str
    box: Box
    op: OpticalParams
    ro: Readout
    tb: TimeBinning
    yield_per_mev: float
    tau_ns: float
    n_events: int
    seed: int
    crystal_name: str
    density: float
    xcom_path: str
    outdir: str


def load_gamma_setup(cfg_path: str, data_dir: Optional[str] = None) -> GammaSetup:
    """The parameters scripts/shoot_gammas.jl:19-45 builds from a run file."""
    with open(cfg_path, "rb") as f:
        cfg = tomllib.load(f)
    data_dir = data_dir or _data_dir_for(cfg_path)
    camp = cfg["campaign"]
    if int(camp["n_events"]) < 1:
        raise ValueError(f"{cfg_path}: campaign.n_events must be >= 1 (got {camp['n_events']})")
    mat = load_material(cfg["crystal"]["material"], data_dir)
    wrap = load_material(cfg["wrap"]["material"], data_dir)
    sipm = load_material(cfg["sipm"]["material"], data_dir)
    sz = [f32(v) for v in cfg["crystal"]["size_mm"]]
    surf = cfg["surface"]
    finish = surf.get("finish", "backpainted")
    op = OpticalParams(f32(mat["n"]), f32(cfg["sipm"]["coupling_n"]), f32(mat["abs_length_mm"]),
                       f32(mat.get("rayleigh_mm", float("inf"))), f32(wrap["reflectivity"]),
                       wrap["model"] == "specular", surface_has_gap(finish),
                       deg2rad_f32(surf["sigma_alpha_deg"]),
                       f32(cfg["sipm"].get("pde_override", sipm["pde"])))
    grid = SipmGrid(f32(sipm["pitch_mm"]), int(sipm["nx"]), int(sipm["ny"]))
    tb = time_binning_from(cfg["binning"])
    xcom = os.path.join(data_dir, cfg["gamma"]["xcom"])
    outdir = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(cfg_path))), "output", camp["tag"])
    return GammaSetup(camp["tag"], cfg, os.path.abspath(cfg_path), Box((sz[0], sz[1], sz[2])), op,
                      Readout(grid), tb, float(mat["yield_per_mev"]), f32(mat["tau_ns"]),
                      int(camp["n_events"]), int(camp["seed"]), mat["name"], float(cfg["gamma"]["density"]),
                      xcom, outdir)


def events_h5_contents(st: GammaSetup, r, backend: str) -> tuple[dict, dict]:
    """Datasets and root attributes of events.h5 (scripts/shoot_gammas.jl:60-78)."""
    datasets = {"edep_kev": r.edep, "npe": r.npe, "maps": r.maps, "tmin_ns": r.tmin,
                "xyz1_mm": r.xyz1, "e1_kev": r.e1, "xyz2_mm": r.xyz2, "e2_kev": r.e2,
                "er_kev": r.er, "int_type": r.int_type, "n_int": r.n_int}
    attrs = {"tag": st.tag, "n_events": np.int64(st.n_events), "seed": np.int64(st.seed),
             "crystal": st.cfg["crystal"]["material"], "pde": np.float32(st.op.pde),
             "backend": backend, "int_type_key": INT_TYPE_KEY, "tmin_nohit": "Inf"}
    return datasets, attrs


def summary(st: GammaSetup, r, elapsed: float, backend: str) -> dict:
    """The printed summary of scripts/shoot_gammas.jl:80-90."""
    n = st.n_events
    interacted = r.edep > 0
    peak = r.edep > np.float32(510.0)
    out = {"tag": st.tag, "n_events": n, "elapsed_s": elapsed, "interacted": float(interacted.mean()),
           "photopeak_fraction": float(peak.mean())}
    print(f"{st.tag:<14s} {n} events ({elapsed:.1f}s, {backend}): interacted "
          f"{100 * interacted.mean():.1f}%, photopeak {100 * peak.mean():.1f}%")
    pe = r.npe[peak].astype(np.float64)
    if pe.size > 0:
        # printed for any photopeak event, as the reference; one event has no
        # sample standard deviation (NaN, as Julia's std)
        m = pe.mean()
        s = pe.std(ddof=1) if pe.size > 1 else float("nan")
        out.update({"photopeak_pe_mean": float(m), "photopeak_fwhm_rel": float(2.355 * s / m)})
        fw = f"{235.5 * s / m:.2f}" if pe.size > 1 else "NaN"
        print(f"{'':<14s} photopeak: {m:.0f} pe mean, FWHM/mean {fw}% "
              "(photostatistics+transport only)")
    return out


def shoot_gammas(cfg_path: str, *, engine=None, surrogate=None, write: bool = True,
                 n_events: Optional[int] = None, data_dir: Optional[str] = None) -> dict:
    """One campaign: events on the GPU, events.h5 under output/<tag>/."""
    from .events import GammaMaterial, run_events
    from .hdf5 import write_h5
    from .transport import default_engine
    st = load_gamma_setup(cfg_path, data_dir)
    if n_events is not None:
        if int(n_events) < 1:
            raise ValueError("n_events must be >= 1")
        st.n_events = int(n_events)
    mat = GammaMaterial.from_csv(st.crystal_name, st.density, st.xcom_path)
    eng = engine or default_engine()
    t0 = time.perf_counter()
    if surrogate is None:
        backend = "cuda"
        r = run_events(st.box, st.op, st.ro, st.tb, mat, st.yield_per_mev, n_events=st.n_events,
                       seed=st.seed, tau_ns=st.tau_ns, engine=eng)
    else:
        backend = "cuda-surrogate"
        r = surrogate.run_events(st.box, st.op, st.ro, st.tb, mat, st.yield_per_mev, n_events=st.n_events,
                                 seed=st.seed, tau_ns=st.tau_ns)
    elapsed = time.perf_counter() - t0
    if write:
        os.makedirs(st.outdir, exist_ok=True)
        shutil.copy(st.cfg_path, os.path.join(st.outdir, os.path.basename(st.cfg_path)))
        datasets, attrs = events_h5_contents(st, r, backend)
        write_h5(os.path.join(st.outdir, "events.h5"), datasets, attrs)
    s = summary(st, r, elapsed, backend)
    s["result"] = r
    return s


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("configs", nargs="+")
    ap.add_argument("--surrogate", default=None, help="trained LightSurrogate (.npz)")
    ap.add_argument("--expert", action="append", default=[],
                    help="depth-slab expert ensemble (.npz) used with --surrogate for the sites "
                         "inside its slab (repeatable)")
    ap.add_argument("--n-events", type=int, default=None, help="override the run file's n_events")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    from .transport import Engine
    eng = Engine(args.device)
    se = None
    if args.surrogate:
        from .fast_events import SurrogateEvents
        from .surrogate import LightSurrogate
        se = SurrogateEvents(LightSurrogate.load(args.surrogate), eng, device=args.device,
                             experts=[LightSurrogate.load(p) for p in args.expert])
    for path in args.configs:
        shoot_gammas(path, engine=eng, surrogate=se, n_events=args.n_events)
    if se is not None:
        se.close()
    eng.close()


if __name__ == "__main__":
    main()
