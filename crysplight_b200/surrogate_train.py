"""Train and validate a light-response surrogate ensemble for one crystal setup.

    python -m crysplight_b200.surrogate_train --setup bgo_esr --out bgo_esr.npz

Steps (all on one GPU):
  1. point scan through the CUDA Monte Carlo: a regular nx x ny x nz grid of
     emission points, ``photons`` photons each, emitted at t = 0 (transit
     times only) with PDE = 1, giving per-SiPM counts and arrival-time moments;
  2. 10% of the grid points are held out; K networks are trained on the rest
     by the library's tcgen05 kernels (Adam, batch 65,536);
  3. held-out validation against a high-statistics Monte Carlo truth on a
     subset of the held-out points: mean per-SiPM relative error of the
     ensemble's detection probabilities over the cells whose expected count at
     ``photons`` photons exceeds 100, next to the same error for the scan table
     itself (each held-out node interpolated from its neighbouring training
     nodes), which is the method without a network.

PDE = 1 in the scan is exact to rescale: the reference detects a photon that
crossed into a SiPM with probability PDE by one last independent draw
(src/transport.jl:161-185), so the detection probability of every SiPM scales
linearly with PDE and the detected photons' times do not depend on it.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .params import Box, OpticalParams, Readout, SipmGrid, deg2rad_f32

# Optical setups of the event campaigns (runs/gammas_csitl_50k.toml with
# data/csitl.toml + data/teflon.toml; runs/gammas_bgo_500k.toml geometry with
# data/bgo.toml + data/esr.toml), PDE 1 for the scan.
SETUPS = {
    "csitl_teflon": dict(box=(48.0, 48.0, 37.2),
                         op=(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, 1.3, 1.0)),
    "bgo_esr": dict(box=(48.0, 48.0, 22.4),
                    op=(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, 1.3, 1.0)),
}


def setup(name: str):
    s = SETUPS[name]
    o = s["op"]
    op = OpticalParams(o[0], o[1], o[2], o[3], o[4], o[5], o[6], deg2rad_f32(o[7]), o[8])
    return Box(s["box"]), op, Readout(SipmGrid(6.0, 8, 8))


def table_interpolate(grid_shape, train_idx, values: np.ndarray, query_idx) -> np.ndarray:
    """The scan table without a network, evaluated at grid nodes that are not
    in the table: per axis, the mean of the two neighbouring nodes when both
    are training nodes (linear interpolation at the midpoint), averaged over
    the axes that have such a pair; nodes with no pair take the mean of
    whichever direct neighbours are training nodes."""
    nx, ny, nz = grid_shape
    have = np.zeros(nx * ny * nz, bool)
    have[train_idx] = True
    q = np.asarray(query_idx)
    ix, iy, iz = q % nx, (q // nx) % ny, q // (nx * ny)
    acc = np.zeros((q.size, values.shape[1]))
    cnt = np.zeros(q.size)
    near = np.zeros((q.size, values.shape[1]))
    ncnt = np.zeros(q.size)
    for axis, (i, n, stride) in enumerate(((ix, nx, 1), (iy, ny, nx), (iz, nz, nx * ny))):
        lo_ok = i > 0
        hi_ok = i < n - 1
        lo = np.where(lo_ok, q - stride, q)
        hi = np.where(hi_ok, q + stride, q)
        lo_ok &= have[lo]
        hi_ok &= have[hi]
        both = lo_ok & hi_ok
        acc[both] += 0.5 * (values[lo[both]] + values[hi[both]])
        cnt += both
        near[lo_ok] += values[lo[lo_ok]]
        near[hi_ok] += values[hi[hi_ok]]
        ncnt += lo_ok.astype(int) + hi_ok.astype(int)
    out = np.where((cnt > 0)[:, None], acc / np.maximum(cnt, 1)[:, None], near / np.maximum(ncnt, 1)[:, None])
    return out


def rel_error(p_pred: np.ndarray, p_true: np.ndarray, photons: int, min_counts: float = 100.0) -> dict:
    """Mean per-SiPM relative error |p - p_true| / p_true over the cells whose
    expected count at ``photons`` photons exceeds ``min_counts``."""
    m = p_true * photons > min_counts
    r = np.abs(p_pred - p_true)[m] / p_true[m]
    return {"mean": float(r.mean()), "median": float(np.median(r)), "p95": float(np.quantile(r, 0.95)),
            "cells": int(m.sum())}


def scan_light_sharded(engine, box, op, ro, pts: np.ndarray, photons: int, seed: int, group):
    """scan_light over the ranks of ``group``: rank r scans a contiguous range
    of the points with the photon ids the single-GPU scan gives them
    (pid_offset = points before x photons), and every rank gets the whole
    result (the same as one GPU's scan)."""
    import torch.distributed as dist
    from .sharding import photon_range
    from .surrogate import ScanResult, scan_light
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    p0, n = photon_range(pts.shape[0], rank, world)
    part = scan_light(engine, box, op, ro, points=pts[p0:p0 + n], photons_per_point=photons, seed=seed,
                      pid_offset=p0 * photons) if n else None
    parts = [None] * world
    dist.all_gather_object(parts, (p0, part), group=group)
    parts = sorted((p for p in parts if p[1] is not None), key=lambda p: p[0])
    cat = lambda f: np.concatenate([getattr(p[1], f) for p in parts], axis=0)
    counters = {}
    for _, r in parts:
        for k, v in r.counters.items():
            counters[k] = counters.get(k, 0) + v
    return ScanResult(pts, photons, cat("counts"), cat("tsum"), cat("tsum2"), cat("tmin"), counters,
                      max(r.seconds for _, r in parts))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--setup", choices=sorted(SETUPS), default="bgo_esr")
    ap.add_argument("--grid", type=int, nargs=3, default=(48, 48, 24))
    ap.add_argument("--photons", type=int, default=100_000)
    ap.add_argument("--members", type=int, default=5)
    ap.add_argument("--steps", type=int, default=20_000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lr-final", type=float, default=1e-5,
                    help="cosine decay of the step size to this value (negative: constant lr)")
    ap.add_argument("--z-warp", type=float, default=0.0,
                    help="depth warp of the grid and of the network input (0 = uniform in z)")
    ap.add_argument("--z-range", type=float, nargs=2, default=None, metavar=("Z0", "Z1"),
                    help="train an expert for the depth slab z0..z1 mm (grid and network input "
                         "span the slab; the event generator uses it for sites inside)")
    ap.add_argument("--first-pass", action="store_true",
                    help="train on the light response minus its first-pass term (cl_surrogate_direct: "
                         "photons that reach the readout face without an interaction), which the "
                         "ensemble adds back exactly; the term carries the sharp pixel edges of "
                         "sites near the readout face")
    ap.add_argument("--compare-model", default=None,
                    help="also validate this ensemble (.npz, e.g. the whole-crystal one) on the "
                         "same held-out points")
    ap.add_argument("--time-weight", type=float, default=0.1,
                    help="loss weight of the arrival-time outputs relative to the probabilities")
    ap.add_argument("--seed", type=int, default=4242)
    ap.add_argument("--truth-points", type=int, default=256)
    ap.add_argument("--truth-photons", type=int, default=10_000_000)
    ap.add_argument("--out", required=True)
    ap.add_argument("--report", default=None)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--model", default=None,
                    help="evaluate this trained ensemble (.npz) instead of training one")
    args = ap.parse_args(argv)

    from .surrogate import LightSurrogate, grid_points, light_targets, scan_light, split_holdout
    from .transport import Engine
    import os

    # under torchrun: one process per GPU; the scan points and the ensemble
    # members are spread over the ranks, rank 0 validates and saves
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    group = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        args.device = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(args.device)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        group = dist.group.WORLD
    box, op, ro = setup(args.setup)
    eng = Engine(args.device)
    rep = {"setup": args.setup, "grid": list(args.grid), "photons_per_point": args.photons,
           "members": args.members, "steps": args.steps, "batch": args.batch, "lr": args.lr,
           "lr_final": args.lr_final, "time_weight": args.time_weight, "z_warp": args.z_warp,
           "z_range": args.z_range}
    pts = grid_points(box, tuple(args.grid), z_warp=args.z_warp, z_range=args.z_range)
    if group is None:
        scan = scan_light(eng, box, op, ro, points=pts, photons_per_point=args.photons, seed=args.seed)
    else:
        scan = scan_light_sharded(eng, box, op, ro, pts, args.photons, args.seed, group)
    n_ph = pts.shape[0] * args.photons
    rep["scan"] = {"points": int(pts.shape[0]), "photons": n_ph, "seconds": scan.seconds,
                   "photons_per_s": n_ph / scan.seconds, "detected_fraction": scan.counters["ndet"] / n_ph}
    print(f"scan: {pts.shape[0]} points x {args.photons} photons in {scan.seconds:.1f} s "
          f"({n_ph / scan.seconds / 1e6:.0f} M photons/s)", flush=True)
    y = light_targets(scan)
    fp = None
    if args.first_pass:
        from .surrogate import FIRST_PASS_FLOOR, first_pass_light, first_pass_optics
        fp = first_pass_optics(op, ro)
        D = first_pass_light(pts, box, fp, args.device).double().cpu().numpy()
        p_scan_all = (scan.counts.astype(np.float64) + 0.5) / (args.photons + 1.0)
        y[:, :64] = np.log(np.maximum(p_scan_all - D, FIRST_PASS_FLOOR)).astype(np.float32)
        rep["first_pass"] = {"mean_sum": float(D.sum(1).mean()),
                             "floored_cells": int((p_scan_all - D < FIRST_PASS_FLOOR).sum())}
    rep["first_pass_optics"] = fp
    tr, ho = split_holdout(pts.shape[0], 0.1, seed=11)
    if args.model:
        sur = LightSurrogate.load(args.model)
    else:
        sur = LightSurrogate.train(box, pts[tr], y[tr], members=args.members, steps=args.steps,
                                   batch=args.batch, lr=args.lr,
                                   lr_final=args.lr_final if args.lr_final >= 0 else None,
                                   time_weight=args.time_weight, z_warp=args.z_warp,
                                   z_range=args.z_range, seed=args.seed,
                                   device=args.device, group=group, first_pass=fp,
                                   log=lambda s: print(s, flush=True))
        rep["train_seconds"] = sur.meta["train_seconds"]
        rep["final_loss"] = [h[-1] for h in sur.meta["loss_history"]]
        print(f"training: {sur.meta['train_seconds']:.1f} s", flush=True)

    if rank != 0:
        eng.close()
        import torch.distributed as dist
        dist.destroy_process_group()
        return rep
    # held-out validation against a high-statistics truth
    rng = np.random.default_rng(5)
    sub = np.sort(rng.choice(ho, size=min(args.truth_points, ho.size), replace=False))
    truth = scan_light(eng, box, op, ro, points=pts[sub], photons_per_point=args.truth_photons,
                       seed=args.seed + 1, batch_points=64)
    p_true = truth.counts / float(args.truth_photons)
    t_true = light_targets(truth)[:, 64:128]
    pred = sur.predict(pts[sub], device=args.device)
    p_scan = scan.counts / float(args.photons)
    p_tab = table_interpolate(tuple(args.grid), tr, p_scan, sub)
    rep["holdout"] = {
        "points": int(sub.size), "truth_photons": args.truth_photons,
        "surrogate": rel_error(pred["p"], p_true, args.photons),
        "members": [rel_error(pm, p_true, args.photons) for pm in pred["p_members"]],
        "table_interpolation": rel_error(p_tab, p_true, args.photons),
        "raw_scan_at_point": rel_error(p_scan[sub], p_true, args.photons),
        "spread_median": float(np.median(pred["spread"])),
        "spread_above_2pct": float(np.mean(pred["spread"] > 0.02)),
        "time_mean_abs_err_ns": float(np.mean(np.abs(pred["t_mean"] - t_true)[p_true * args.photons > 100])),
        "spread_p95": float(np.quantile(pred["spread"], 0.95)),
        "truth_noise_mean": float(np.mean(np.sqrt(1.0 / np.maximum(truth.counts[p_true * args.photons > 100], 1)))),
    }
    # the points the surrogate serves in event generation: at least 1 mm from a
    # wrapped face (the four sides and the front face z = 0) and spread <= 2%
    q = pts[sub].astype(np.float64)
    L = [float(box.L[i]) for i in range(3)]
    d_wall = np.minimum.reduce([q[:, 0], L[0] - q[:, 0], q[:, 1], L[1] - q[:, 1], q[:, 2]])
    served = (d_wall >= 1.0) & (pred["spread"] <= 0.02)
    rep["holdout"]["served_points"] = int(served.sum())
    rep["holdout"]["surrogate_served"] = rel_error(pred["p"][served], p_true[served], args.photons)
    rep["holdout"]["table_served"] = rel_error(p_tab[served], p_true[served], args.photons)
    far = d_wall >= 1.0
    rep["holdout"]["surrogate_wall_ge_1mm"] = rel_error(pred["p"][far], p_true[far], args.photons)
    per_pt = np.array([rel_error(pred["p"][i:i + 1], p_true[i:i + 1], args.photons)["mean"]
                       for i in range(sub.size)])
    dz_read = L[2] - q[:, 2]
    rep["holdout"]["by_distance_to_readout_mm"] = {
        f"{lo}-{hi}": float(per_pt[(dz_read >= lo) & (dz_read < hi)].mean())
        for lo, hi in ((0, 2), (2, 5), (5, 10), (10, 30)) if ((dz_read >= lo) & (dz_read < hi)).any()}
    bins_read = ((0, 1), (1, 2), (2, 4), (4, 8), (8, 30))
    rep["holdout"]["spread_above_2pct_by_distance_to_readout_mm"] = {
        f"{lo}-{hi}": float(np.mean(pred["spread"][(dz_read >= lo) & (dz_read < hi)] > 0.02))
        for lo, hi in bins_read if ((dz_read >= lo) & (dz_read < hi)).any()}
    if args.compare_model:
        other = LightSurrogate.load(args.compare_model).predict(pts[sub], device=args.device)
        per_o = np.array([rel_error(other["p"][i:i + 1], p_true[i:i + 1], args.photons)["mean"]
                          for i in range(sub.size)])
        rep["holdout"]["compare_model"] = {
            "path": args.compare_model, "surrogate": rel_error(other["p"], p_true, args.photons),
            "by_distance_to_readout_mm": {
                f"{lo}-{hi}": float(per_o[(dz_read >= lo) & (dz_read < hi)].mean())
                for lo, hi in bins_read if ((dz_read >= lo) & (dz_read < hi)).any()},
            "spread_above_2pct_by_distance_to_readout_mm": {
                f"{lo}-{hi}": float(np.mean(other["spread"][(dz_read >= lo) & (dz_read < hi)] > 0.02))
                for lo, hi in bins_read if ((dz_read >= lo) & (dz_read < hi)).any()}}
        rep["holdout"]["surrogate_by_distance_to_readout_mm_fine"] = {
            f"{lo}-{hi}": float(per_pt[(dz_read >= lo) & (dz_read < hi)].mean())
            for lo, hi in bins_read if ((dz_read >= lo) & (dz_read < hi)).any()}
    rep["holdout"]["by_distance_to_wall_mm"] = {
        f"{lo}-{hi}": float(per_pt[(d_wall >= lo) & (d_wall < hi)].mean())
        for lo, hi in ((0, 1), (1, 3), (3, 8), (8, 30)) if ((d_wall >= lo) & (d_wall < hi)).any()}
    print(json.dumps(rep["holdout"], indent=1), flush=True)
    if args.model:
        if args.report:
            with open(args.report, "w") as f:
                json.dump(rep, f, indent=1)
        eng.close()
        if group is not None:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rep
    sur.meta.update({"setup": args.setup, "grid": list(args.grid), "photons_per_point": args.photons,
                     "z_range": args.z_range, "first_pass": fp})
    sur.save(args.out)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    eng.close()
    if group is not None:
        import torch.distributed as dist
        dist.destroy_process_group()
    return rep


if __name__ == "__main__":
    main()
