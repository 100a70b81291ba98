"""Run summary and output files (src/output.jl).

``write_output`` mirrors src/output.jl:4-52: the printed summary, the 8-fold
symmetry residual, and ``output/<tag>/light.h5`` plus a copy of the run file.
"""
from __future__ import annotations

import os
import shutil

import numpy as np

from .params import Accumulator


def symmetry_residual(m: np.ndarray) -> float:
    """src/output.jl:58-62: max relative deviation of a map from its 8-fold
    symmetrisation (x-mirror, y-mirror, transpose)."""
    m = np.asarray(m, dtype=np.float64)
    mt = m.T
    ms = (m + m[::-1, :] + m[:, ::-1] + m[::-1, ::-1]
          + mt + mt[::-1, :] + mt[:, ::-1] + mt[::-1, ::-1]) / 8.0
    return float(np.max(np.abs(m - ms) / np.maximum(ms, 1.0)))


def summary(st, acc: Accumulator, elapsed: float) -> dict:
    n = st.n_photons
    m = acc.counts.sum(axis=2, dtype=np.int64)
    mean_bounces = acc.sum_bounces_det / acc.ndet if acc.ndet > 0 else float("nan")
    return {
        "tag": st.tag, "n_photons": n, "detected_fraction": acc.ndet / n,
        "abs_bulk_fraction": acc.nabs_bulk / n, "abs_wall_fraction": acc.nabs_wall / n,
        "abs_sipm_fraction": acc.nabs_sipm / n, "cap_fraction": acc.ncap / n,
        "mean_bounces_detected": mean_bounces, "symmetry_residual": symmetry_residual(m),
        "elapsed_s": elapsed,
    }


def light_h5_contents(st, acc: Accumulator) -> tuple[dict, dict]:
    """Datasets and root attributes of light.h5 (src/output.jl:10-32)."""
    surf = st.cfg.get("surface", {})
    datasets = {"counts": acc.counts, "first_time_ns": acc.first_ns}
    attrs = {
        "tag": st.tag, "n_photons": np.int64(st.n_photons), "seed": np.int64(st.seed),
        "bin_ns": np.float32(st.tb.bin_ns), "nbins": np.int32(st.tb.nbins),
        "crystal": st.cfg["crystal"]["material"], "wrap": st.cfg["wrap"]["material"],
        "pde": np.float32(st.op.pde), "ndet": np.int64(acc.ndet),
        "nabs_bulk": np.int64(acc.nabs_bulk), "nabs_wall": np.int64(acc.nabs_wall),
        "nabs_sipm": np.int64(acc.nabs_sipm), "ncap": np.int64(acc.ncap),
        "nabs_surround": np.int64(acc.nabs_sur), "nscat": np.int64(acc.nscat),
        "finish": surf.get("finish", "backpainted"),
        "sigma_alpha_deg": np.float64(surf.get("sigma_alpha_deg", 0.0)),
    }
    return datasets, attrs


def write_output(st, acc: Accumulator, elapsed: float, write: bool = True) -> dict:
    s = summary(st, acc, elapsed)
    if write:
        from .hdf5 import write_h5
        os.makedirs(st.outdir, exist_ok=True)
        shutil.copy(st.cfg_path, os.path.join(st.outdir, os.path.basename(st.cfg_path)))
        datasets, attrs = light_h5_contents(st, acc)
        write_h5(os.path.join(st.outdir, "light.h5"), datasets, attrs)
    n = st.n_photons
    print(f"{st.tag:<22s}  detected {100 * s['detected_fraction']:6.2f}%   bulk "
          f"{100 * acc.nabs_bulk / n:6.2f}%   wall {100 * acc.nabs_wall / n:6.2f}%   cap "
          f"{acc.ncap / n:.2e}")
    print(f"{'':<22s}  <bounces|det> {s['mean_bounces_detected']:.1f}   symmetry residual "
          f"{s['symmetry_residual']:.3f}   {elapsed:.2f}s (CUDA)")
    return s
