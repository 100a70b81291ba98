#!/usr/bin/env python
"""Throughput of the B200 optical-photon transport.

Workload (one "step" = one pass over it):
  scan256  (default) BGO + ESR crystal 48x48x22.4 mm, 256 emission points
           uniform in the volume (Philox key 7), 200,000 isotropic photons per
           point = 51.2M photons, per-point 8x8 count and first-hit maps.
  point1m  CsI(Tl) + Teflon 48x48x37.2 mm, 1,000,000 photons from the centre,
           8x8x81 count histogram and 8x8 first-hit map.
  events_csitl          50,000 511 keV gammas on CsI(Tl) + Teflon: events/s.
  events_bgo_surrogate  500,000 511 keV gammas on BGO + ESR through the
           learned surrogate with Monte Carlo fallback, against the plain
           Monte Carlo of the same events: events/s.

The default run adds secondary objects to its line: the 511 keV events/s of
the event pipeline (a 10,000-event sample of events_csitl, --events), the
surrogate MLP's training throughput on the tensor cores
(--surrogate-training), and events_bgo_surrogate (--surrogate-events).

Arms:
  --impl cuda       (default) the sm_100a library; `value` = photons/s with
                    inputs resident in HBM (device entry point, CUDA events on
                    the launch stream, L2 flushed between steps); `e2e` =
                    photons/s through the host-buffer C-ABI call (pinned host
                    inputs copied in, maps/times/counters copied out).
  --impl reference  the CPU restatement of the reference's transport
                    (oracle/, all host threads) on a bounded sample of the
                    same workload; the reference itself is Julia, absent here.

Multi-GPU (torchrun): every rank transports its own full workload with a
disjoint photon-id range (weak scaling, no data-path collective); the time is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np

# Reference operations per photon-step (Float32/int arithmetic of the reference's
# transport expressions, log/sin/cos/sqrt/div one each), counted by the
# instrumented oracle (python -m oracle.opcount).
OPS_PER_STEP = {"scan256": 165.6, "point1m": 186.7}
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (read + write) per launch of the transport kernel: one ncu capture
# of the scan at 20,000 photons per point (profiles/transport_kernel_scan256x20k.md,
# 3.00 GB for 494.8M photon-steps) scaled to the full launch by photon-steps.
# Almost all of it is L2 misses of the 64 MB log table (about 2 bytes per
# photon-step x log lookup), which grow in proportion to the steps; the
# sources, offsets and maps are 0.24 MB.  point1m: not captured.
TRAFFIC_PER_STEP = (2.993991e9 + 6.48064e6) / 494_804_727
TRAFFIC_BYTES = {"point1m": None}
# Warp instructions the transport kernel issues per photon-step (smsp__inst_executed
# of the same ncu capture: 17.23 G for 494.8M photon-steps); with the live
# steps/s this gives the kernel's issue rate against the SMs' issue slots.
WARP_INST_PER_STEP = {"scan256": 17228482017 / 494_804_727}


def events_workload(n_events: int = 50_000):
    """511 keV gammas on CsI(Tl) + Teflon (runs/gammas_csitl_50k.toml:
    seed 11, PDE 0.40, 100 ns x 80 bins, yield 54000/MeV, tau 1000 ns)."""
    from crysplight_b200.params import (Box, OpticalParams, Readout, SipmGrid, TimeBinning,
                                        deg2rad_f32)
    from crysplight_b200.events import GammaMaterial
    box = Box((48.0, 48.0, 37.2))
    op = OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, deg2rad_f32(1.3), 0.40)
    return dict(name="events_csitl", box=box, op=op, ro=Readout(SipmGrid(6.0, 8, 8)),
                tb=TimeBinning(100.0, 80), tau=1000.0, seed=11, yield_=54_000.0,
                mat=GammaMaterial.from_csv("CsI", 4.51, "xcom_CSI.csv"), n_events=n_events,
                desc=f"{n_events} 511 keV gammas, CsI(Tl)+Teflon 48x48x37.2 mm, PDE 0.40")


def run_events_bench(eng, E, steps: int, warmup: int, dev, stream, pid_base: int = 0):
    """events/s: the transport of all events' photons with the deposits in HBM
    (value: one CUDA-graph replay of init + transport + finalize per step, at
    the launch shape the autotuner picked), and the whole public pipeline
    run_events (e2e)."""
    import torch
    from crysplight_b200.batching import DeviceEvents, autotune
    from crysplight_b200.events import gamma_stage, run_events
    g = gamma_stage(E["mat"], E["box"], n_events=E["n_events"], seed=E["seed"],
                    yield_per_mev=E["yield_"])
    nd = g.dep_photons.size
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n_seg = E["n_events"]
    ev = DeviceEvents(eng, E["box"], E["op"], E["ro"], E["tb"], xyz=T(g.dep_xyz), t0=T(g.dep_t),
                      photons=T(g.dep_photons), segment=T(g.dep_event), n_segments=n_seg,
                      seed=E["seed"], tau_ns=E["tau"], pid_offset=pid_base)
    best, tune_times = autotune(eng, ev.step, stream=stream, repeats=2)
    ev.capture()
    for _ in range(warmup):
        ev.replay()
    ev.sync(stream)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    marks = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(steps)]
    for a, b in marks:
        flush.zero_()
        a.record(stream)
        ev.replay()
        b.record(stream)
    ev.sync(stream)
    dev_s = sum(a.elapsed_time(b) for a, b in marks) * 1e-3 / steps
    photon_steps = eng.last_steps
    run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"],
               n_events=E["n_events"], seed=E["seed"], tau_ns=E["tau"], engine=eng)
    t0 = time.perf_counter()
    for _ in range(steps):
        run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"],
                   n_events=E["n_events"], seed=E["seed"], tau_ns=E["tau"], engine=eng)
    e2e_s = (time.perf_counter() - t0) / steps
    eng.set_launch(0, 0, 0)
    return dict(value=E["n_events"] / dev_s, e2e=E["n_events"] / e2e_s, dev_s=dev_s,
                e2e_s=e2e_s, photons=ev.n_photons, photon_steps=photon_steps, deposits=nd,
                launch={"ctas_per_sm": best.ctas_per_sm, "threads_per_cta": best.threads_per_cta,
                        "warp_chunk": best.warp_chunk},
                tune_ms={f"{k.threads_per_cta}x{k.ctas_per_sm}/{k.warp_chunk}": round(v * 1e3, 3)
                         for k, v in tune_times.items()},
                h2d=int(3 * 4 * nd + 4 * nd + 8 * nd + 4 * nd),
                d2h=int(2 * 4 * 64 * n_seg + 4 * n_seg + 72 + 12))


def surrogate_training_bench(dev, steps: int = 200, warmup: int = 20) -> dict:
    """Adam steps of the surrogate MLP (3->256->256->256->192, batch 65,536) on
    the tcgen05 kernels, synthetic training data: ms per step and TFLOP/s
    against the measured dense BF16 peak (sustained: a long loop)."""
    import torch
    from crysplight_b200.surrogate import MLP
    n = 55_296
    g = torch.Generator(device=dev).manual_seed(3)
    x = torch.rand(n, 3, device=dev, generator=g) * 2 - 1
    t = torch.randn(n, 192, device=dev, generator=g)
    m = MLP(dev.index or 0, max_batch=65536, seed=1)
    m.set_data(x, t)
    m.train(warmup, batch=65536)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    m.train(steps, batch=65536)
    torch.cuda.synchronize(dev)
    dt = (time.perf_counter() - t0) / steps
    m.close()
    flop = 65536 * 2 * 3 * (3 * 256 + 2 * 256 * 256 + 256 * 192)      # forward + 2 x backward
    peak = measured_peaks().get("bf16_tflops_sustained", 1400.0)
    return {"metric": "surrogate training steps/s", "batch": 65536, "ms_per_step": dt * 1e3,
            "tflops": flop / dt / 1e12, "peak_tflops": peak, "frac": flop / dt / 1e12 / peak,
            "note": "one cl_mlp_train call of all steps (host time around a synchronised loop)"}


SURROGATE_BGO = os.path.join(ROOT, "crysplight_b200", "surrogates", "bgo_esr.npz")
# the expert ensemble of the last millimetres before the readout face (used when present)
SURROGATE_BGO_FACE = os.path.join(ROOT, "crysplight_b200", "surrogates", "bgo_esr_face.npz")


def surrogate_events_workload(n_events: int = 500_000):
    """511 keV gammas on BGO + ESR (geometry of runs/gammas_bgo_500k.toml,
    48x48x22.4 mm, PDE 0.40, 100 ns x 120 bins; seed 99, yield 14000/MeV,
    tau 1768 ns, density 7.13 g/cm3)."""
    from crysplight_b200.params import (Box, OpticalParams, Readout, SipmGrid, TimeBinning,
                                        deg2rad_f32)
    from crysplight_b200.events import GammaMaterial
    box = Box((48.0, 48.0, 22.4))
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, deg2rad_f32(1.3), 0.40)
    return dict(name="events_bgo_surrogate", box=box, op=op, ro=Readout(SipmGrid(6.0, 8, 8)),
                tb=TimeBinning(100.0, 120), tau=1768.0, seed=99, yield_=14_000.0,
                mat=GammaMaterial.from_csv("BGO", 7.13, "xcom_BGO.csv"), n_events=n_events,
                desc=f"{n_events} 511 keV gammas, BGO+ESR 48x48x22.4 mm, PDE 0.40, surrogate "
                     "light maps with Monte Carlo fallback (ensemble spread > 2% or < 1 mm "
                     "from a wrapped face)")


def run_surrogate_events_bench(eng, E, steps: int, warmup: int, dev, stream, wall_min_mm=1.0,
                               expert: bool = True):
    """events/s of the surrogate + fallback pipeline with the deposits in HBM
    (value), the plain Monte Carlo on the same deposits, their agreement, and
    the whole public call SurrogateEvents.run_events (e2e)."""
    import torch
    from crysplight_b200.events import gamma_stage
    from crysplight_b200.fast_events import SurrogateEvents, compare_maps, photopeak
    from crysplight_b200.surrogate import LightSurrogate
    sur = LightSurrogate.load(SURROGATE_BGO)
    experts = [LightSurrogate.load(SURROGATE_BGO_FACE)] if expert and os.path.exists(SURROGATE_BGO_FACE) else []
    se = SurrogateEvents(sur, eng, device=dev.index or 0, experts=experts)
    g = gamma_stage(E["mat"], E["box"], n_events=E["n_events"], seed=E["seed"],
                    yield_per_mev=E["yield_"])
    nd = g.dep_photons.size
    n_seg = E["n_events"]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    xyz, t0, ph, seg = T(g.dep_xyz), T(g.dep_t), T(g.dep_photons), T(g.dep_event)
    sptr = stream.cuda_stream
    kw = dict(xyz=xyz, t0=t0, photons=ph, segment=seg, n_segments=n_seg, seed=E["seed"],
              tau_ns=E["tau"], wall_min_mm=wall_min_mm, stream=sptr)

    def step():
        return se.transport_sites(E["box"], E["op"], E["ro"], E["tb"], **kw)
    for _ in range(warmup):
        step()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    times, out = [], None
    for _ in range(steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = step()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b) * 1e-3)
    (maps, tmin, npe, ctr, sampled), stats = out
    dev_s = sum(times) / steps
    s_maps = maps.cpu().numpy().view(np.uint32).reshape(n_seg, 64)
    s_npe = npe.cpu().numpy()
    # the plain Monte Carlo of every deposit
    off = np.zeros(nd + 1, np.int64)
    np.cumsum(g.dep_photons, out=off[1:])
    d_off = T(off)
    m_maps = torch.empty(64 * n_seg, dtype=torch.int32, device=dev)
    m_tmin = torch.empty(64 * n_seg, dtype=torch.float32, device=dev)
    m_npe = torch.empty(n_seg, dtype=torch.int32, device=dev)
    m_ctr = torch.empty(9, dtype=torch.int64, device=dev)
    xs = [xyz[:, i].contiguous() for i in range(3)]
    flush.zero_()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    eng.run_segments_device(E["box"], E["op"], E["ro"], E["tb"], sx=xs[0].data_ptr(),
                            sy=xs[1].data_ptr(), sz=xs[2].data_ptr(), st=t0.data_ptr(),
                            src_offsets=d_off.data_ptr(), src_segment=seg.data_ptr(), n_src=nd,
                            n_segments=n_seg, n_photons=int(off[-1]), seed=E["seed"] + 1,
                            pid_offset=0, tau_ns=E["tau"], maps=m_maps.data_ptr(),
                            tmin=m_tmin.data_ptr(), npe=m_npe.data_ptr(), counters=m_ctr.data_ptr(),
                            stream=sptr)
    b.record(stream)
    eng.sync(sptr)
    mc_s = a.elapsed_time(b) * 1e-3
    mc_steps = eng.last_steps
    mm = m_maps.cpu().numpy().view(np.uint32).reshape(n_seg, 64)
    pk_s, pk_m = photopeak(s_npe, g.edep), photopeak(m_npe.cpu().numpy(), g.edep)
    cmp = compare_maps(s_maps.T.reshape(8, 8, n_seg), mm.T.reshape(8, 8, n_seg))
    # end to end: the public call (host gamma stage, copies in, maps out)
    se.run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"], n_events=n_seg,
                  seed=E["seed"], tau_ns=E["tau"], wall_min_mm=wall_min_mm)
    t_e2e = time.perf_counter()
    for _ in range(steps):
        se.run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"], n_events=n_seg,
                      seed=E["seed"], tau_ns=E["tau"], wall_min_mm=wall_min_mm)
    e2e_s = (time.perf_counter() - t_e2e) / steps
    # our kernels per step: per ensemble, inputs + K members x 65536-row chunks
    # x (layer 1 + 3 tcgen05 GEMMs) + combine; then init + transport + sampler + finalize
    chunks = lambda n: -(-int(n) // 65536)
    launches = 2 + len(sur.members) * chunks(nd) * 4 + 4
    for e in experts:
        z0, z1 = e.depth_range()
        ne = int(np.count_nonzero((g.dep_xyz[:, 2] >= z0 + se.expert_margin_mm) & (g.dep_xyz[:, 2] <= z1)))
        launches += (2 + len(e.members) * chunks(ne) * 4) if ne else 0
    se.close()
    return dict(value=n_seg / dev_s, e2e=n_seg / e2e_s, dev_s=dev_s, mc_value=n_seg / mc_s,
                mc_s=mc_s, mc_photon_steps=mc_steps, photons=int(off[-1]), deposits=nd,
                members=len(sur.members), experts=len(experts), launches=launches,
                stats=stats, photopeak_surrogate=pk_s, photopeak_mc=pk_m,
                photopeak_shift=(pk_s["mean"] - pk_m["mean"]) / pk_m["mean"], maps=cmp,
                h2d=int(12 * nd + 4 * nd + 8 * nd + 4 * nd), d2h=int(2 * 4 * 64 * n_seg + 4 * n_seg + 72 + 16 + nd))


def events_cpu_baseline(E, target_s: float) -> dict:
    """The oracle transports the photons of a sample of events (after the host
    gamma stage) on all host threads: events/s."""
    from oracle import oracle
    from crysplight_b200.events import gamma_stage
    n = 50
    while True:
        g = gamma_stage(E["mat"], E["box"], n_events=n, seed=E["seed"], yield_per_mev=E["yield_"])
        t0 = time.perf_counter()
        oracle.run_segments(E["box"], E["op"], E["ro"], E["tb"], sources=g.dep_xyz,
                            photons_per_source=g.dep_photons, segment_of_source=g.dep_event,
                            n_segments=n, seed=E["seed"], t0s=g.dep_t, tau_ns=E["tau"],
                            nthreads=os.cpu_count())
        dt = time.perf_counter() - t0
        if dt > 0.3 * target_s or n >= E["n_events"]:
            break
        n = min(E["n_events"], int(n * max(2.0, target_s / max(dt, 1e-3))))
    return {"value": n / dt, "unit": "events/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"first {n} of the {E['n_events']} events ({dt:.1f} s on "
                      f"{os.cpu_count()} threads; gamma stage excluded)"}


def issue_slots(name: str, steps_per_s: float, n_sm: int, sm_mhz: float):
    """The transport kernel's warp-instruction issue rate (warp instructions
    per photon-step from the committed ncu capture x the live photon-steps/s)
    against the SMs' issue slots (4 schedulers per SM, one instruction per
    clock each, at the max SM clock); None where no capture exists."""
    wi = WARP_INST_PER_STEP.get(name)
    if wi is None:
        return None
    achieved = wi * steps_per_s
    peak = n_sm * 4 * sm_mhz * 1e6
    return {"achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "G warp-instructions/s",
            "frac": achieved / peak, "warp_inst_per_step": wi}


def workload(name: str, points: int = 256, per_point: int = 200_000):
    from crysplight_b200.params import (Box, OpticalParams, Readout, SipmGrid, TimeBinning,
                                        deg2rad_f32)
    from crysplight_b200.scan import scan_points
    grid, tb = SipmGrid(6.0, 8, 8), TimeBinning(100.0, 80)
    if name == "scan256":
        box = Box((48.0, 48.0, 22.4))
        op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, deg2rad_f32(1.3), 1.0)
        pts = scan_points(256, box, seed=7)[:points]
        return dict(name=name, box=box, op=op, ro=Readout(grid), tb=tb, tau=1768.0, seed=1234,
                    points=pts, per_point=per_point, n=points * per_point,
                    desc=f"BGO+ESR 48x48x22.4 mm, {points} points x {per_point} photons, "
                         "per-point 8x8 maps")
    box = Box((48.0, 48.0, 37.2))
    op = OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, deg2rad_f32(1.3), 1.0)
    return dict(name=name, box=box, op=op, ro=Readout(grid), tb=tb, tau=1000.0, seed=1234,
                points=np.float32([[24.0, 24.0, 18.6]]), per_point=1_000_000, n=1_000_000,
                desc="CsI(Tl)+Teflon 48x48x37.2 mm, 1e6 photons from the centre, 8x8x81 histogram")


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"cl_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        busy = [v for v in sm if smax and v > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "fallback": True}


# ------------------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle on the host cores
# ------------------------------------------------------------------------------------
def cpu_run(W, n_points: int, per_point: int) -> tuple[float, int]:
    from oracle import oracle
    pts = W["points"][:n_points]
    t0 = time.perf_counter()
    if W["name"] == "scan256":
        oracle.run_segments(W["box"], W["op"], W["ro"], W["tb"], sources=pts,
                            photons_per_source=[per_point] * n_points,
                            segment_of_source=range(n_points), n_segments=n_points,
                            seed=W["seed"], tau_ns=W["tau"], nthreads=os.cpu_count())
    else:
        oracle.run_photons(W["box"], W["op"], W["ro"], W["tb"], n_photons=per_point,
                           seed=W["seed"], pos=tuple(pts[0]), tau_ns=W["tau"],
                           nthreads=os.cpu_count())
    dt = time.perf_counter() - t0
    return dt, n_points * per_point


def cpu_sample_size(W, target_s: float) -> tuple[int, int]:
    """(points, photons per point) of a sample that takes about target_s."""
    if W["name"] == "scan256":
        dt, n = cpu_run(W, 1, 20_000)
        pts = int(max(1, min(256, target_s / (dt * W["per_point"] / 20_000))))
        return pts, W["per_point"]
    dt, n = cpu_run(W, 1, 50_000)
    per = int(max(50_000, min(W["per_point"] * 50, target_s / dt * 50_000)))
    return 1, per


def cpu_baseline(W, target_s: float) -> dict:
    pts, per = cpu_sample_size(W, target_s)
    dt, n = cpu_run(W, pts, per)
    return {"value": n / dt, "unit": "photons/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{pts} point(s) x {per} photons of the {W['name']} workload "
                      f"({dt:.1f} s on {os.cpu_count()} threads)"}


def run_reference_arm(args, W, rank, world):
    if rank != 0:
        return
    pts, per = cpu_sample_size(W, args.cpu_seconds)
    for _ in range(args.warmup):
        cpu_run(W, pts, per)
    times = []
    for _ in range(args.steps):
        dt, n = cpu_run(W, pts, per)
        times.append(dt)
    tot_n = n * args.steps
    value = tot_n / sum(times)
    sample = (f"{pts} point(s) x {per} photons of the {W['name']} workload per step "
              f"(C restatement of the reference CPU transport, {os.cpu_count()} threads)")
    line = {
        "impl": "reference", "metric": "photons/s", "value": value, "unit": "photons/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": W["name"], "desc": W["desc"], "sample_photons_per_step": n},
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------
# CUDA arm
# ------------------------------------------------------------------------------------
def run_cuda_arm(args, W, rank, world, local_rank):
    import torch
    import crysplight_b200 as cl
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    eng = cl.Engine(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

    pid_base = rank * W["n"]        # disjoint photon ids per rank
    stream = torch.cuda.Stream(dev)  # explicit stream: the library launches on it
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    nx = ny = 8
    pts = W["points"]
    npts = pts.shape[0]
    if W["name"] == "scan256":
        off = np.zeros(npts + 1, np.int64)
        off[1:] = np.cumsum(np.full(npts, W["per_point"], np.int64))
        seg = np.arange(npts, dtype=np.int32)
        d_sx = torch.from_numpy(np.ascontiguousarray(pts[:, 0])).to(dev)
        d_sy = torch.from_numpy(np.ascontiguousarray(pts[:, 1])).to(dev)
        d_sz = torch.from_numpy(np.ascontiguousarray(pts[:, 2])).to(dev)
        d_off = torch.from_numpy(off).to(dev)
        d_seg = torch.from_numpy(seg).to(dev)
        d_maps = torch.empty(nx * ny * npts, dtype=torch.int32, device=dev)
        d_tmin = torch.empty(nx * ny * npts, dtype=torch.float32, device=dev)
        d_npe = torch.empty(npts, dtype=torch.int32, device=dev)
        d_ctr = torch.empty(9, dtype=torch.int64, device=dev)

        def device_step():
            eng.run_segments_device(
                W["box"], W["op"], W["ro"], W["tb"], sx=d_sx.data_ptr(), sy=d_sy.data_ptr(),
                sz=d_sz.data_ptr(), st=None, src_offsets=d_off.data_ptr(),
                src_segment=d_seg.data_ptr(), n_src=npts, n_segments=npts, n_photons=W["n"],
                seed=W["seed"], pid_offset=pid_base, tau_ns=W["tau"], maps=d_maps.data_ptr(),
                tmin=d_tmin.data_ptr(), npe=d_npe.data_ptr(), counters=d_ctr.data_ptr(),
                stream=sptr)

        # pinned host inputs for the end-to-end path
        h_pts = torch.from_numpy(np.ascontiguousarray(pts)).pin_memory().numpy()
        h_cnt = torch.full((npts,), W["per_point"], dtype=torch.int64).pin_memory().numpy()
        h_seg = torch.from_numpy(seg).pin_memory().numpy()

        def host_step():
            return eng.run_segments(W["box"], W["op"], W["ro"], W["tb"], sources=h_pts,
                                    photons_per_source=h_cnt, segment_of_source=h_seg,
                                    n_segments=npts, seed=W["seed"], pid_offset=pid_base,
                                    tau_ns=W["tau"])
        h2d = 3 * 4 * npts + 8 * (npts + 1) + 4 * npts
        d2h = 2 * 4 * nx * ny * npts + 4 * npts + 72 + 12
        out_bytes = 2 * 4 * nx * ny * npts + 4 * npts + 72
        launches = 3
    else:
        d_p = [torch.from_numpy(np.ascontiguousarray(pts[:, i])).to(dev) for i in range(3)]
        nb = W["tb"].nbins + 1
        d_counts = torch.empty(nx * ny * nb, dtype=torch.int32, device=dev)
        d_first = torch.empty(nx * ny, dtype=torch.float32, device=dev)
        d_ctr = torch.empty(9, dtype=torch.int64, device=dev)

        def device_step():
            eng.run_photons_device(W["box"], W["op"], W["ro"], W["tb"], px=d_p[0].data_ptr(),
                                   py=d_p[1].data_ptr(), pz=d_p[2].data_ptr(), pt=None, npos=1,
                                   n_photons=W["n"], seed=W["seed"], pid_offset=pid_base,
                                   tau_ns=W["tau"], counts=d_counts.data_ptr(),
                                   first_ns=d_first.data_ptr(), counters=d_ctr.data_ptr(),
                                   stream=sptr)
        h_pos = tuple(float(v) for v in pts[0])

        def host_step():
            return eng.run_photons_ka(W["box"], W["op"], W["ro"], W["tb"], n_photons=W["n"],
                                      seed=W["seed"], pos=h_pos, pid_offset=pid_base,
                                      tau_ns=W["tau"])
        h2d = 3 * 4
        d2h = 4 * nx * ny * nb + 4 * nx * ny + 72 + 12
        out_bytes = 4 * nx * ny * nb + 4 * nx * ny + 72
        launches = 2

    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # warm-up
    for _ in range(args.warmup):
        device_step()
    eng.sync(sptr)
    host_step()

    # ---- device-resident timing ----
    clocks = ClockSampler(local_rank)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    clocks.start()
    t_wall0 = time.perf_counter()
    for i in range(args.steps):
        flush.zero_()                       # evict L2 between timed steps
        starts[i].record(stream)
        device_step()
        stops[i].record(stream)
    eng.sync(sptr)
    barrier()
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, stops)]
    steps_per_launch = eng.last_steps
    tot_ms = sum(step_ms)

    # ---- end-to-end through the host-buffer C-ABI ----
    barrier()
    e2e_t0 = time.perf_counter()
    for _ in range(args.steps):
        host_step()
    barrier()
    e2e_s = time.perf_counter() - e2e_t0

    if dist is not None:
        t = torch.tensor([tot_ms, e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms, e2e_s = float(t[0]), float(t[1])

    if rank != 0:
        eng.close()
        return
    n_total = W["n"] * args.steps * world
    value = n_total / (tot_ms * 1e-3)
    e2e_value = n_total / e2e_s
    peaks = measured_peaks()
    props = torch.cuda.get_device_properties(dev)
    n_sm = props.multi_processor_count
    launch_s = tot_ms * 1e-3 / args.steps
    ops_step = OPS_PER_STEP[W["name"]]
    achieved = ops_step * steps_per_launch / launch_s
    peak = n_sm * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6
    line = {
        "metric": "photons/s", "value": value, "unit": "photons/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": W["name"], "desc": W["desc"], "photons_per_step_per_gpu": W["n"],
                   "l2": "flushed between timed steps (256 MiB memset)",
                   "parallelism": f"photon-range shards x{world}"},
        "e2e": {"value": e2e_value, "unit": "photons/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches * args.steps,
        "photon_steps_per_launch": steps_per_launch,
        "photon_steps_per_s": steps_per_launch / launch_s,
        "roofline": {
            "bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gop/s",
            "frac": achieved / peak,
            "traffic": (TRAFFIC_PER_STEP * steps_per_launch if W["name"] == "scan256"
                        else TRAFFIC_BYTES.get(W["name"])),
            "ops_per_step": ops_step,
            "note": ("reference Float32/int ops per photon-step x steps / launch time, against "
                     "one op per lane per clock (SMs x 128 lanes x max SM clock of measured)"),
            "hbm": {"achieved": out_bytes / launch_s / 1e9, "peak": peaks.get("hbm_gbs"),
                    "unit": "GB/s", "frac": out_bytes / launch_s / 1e9 / peaks.get("hbm_gbs", 1)},
            "issue_slots": issue_slots(W["name"], steps_per_launch / launch_s, n_sm,
                                       peaks.get("sm_max_mhz", 1965.0)),
        },
        "clocks": clk,
        "wall_s_timed": t_wall,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(W, args.cpu_seconds)
    if world == 1 and args.events > 0:
        # secondary metric: 511 keV events/s of the event pipeline (10,000 CsI(Tl) events)
        E = events_workload(args.events)
        r = run_events_bench(eng, E, args.steps, args.warmup, dev, stream)
        line["events"] = {"metric": "511keV events/s", "workload": E["desc"],
                          "value": r["value"], "e2e": r["e2e"], "unit": "events/s",
                          "photons_per_event": r["photons"] / E["n_events"],
                          "photon_steps_per_s": r["photon_steps"] / r["dev_s"],
                          "launch": r["launch"], "cuda_graph": True}
    if world == 1 and args.surrogate_training:
        line["surrogate_training"] = surrogate_training_bench(dev)
    if world == 1 and args.surrogate_events > 0 and os.path.exists(SURROGATE_BGO):
        # secondary metric: 500,000 BGO+ESR events, surrogate + Monte Carlo fallback vs
        # the plain Monte Carlo
        E = surrogate_events_workload(args.surrogate_events)
        r = run_surrogate_events_bench(eng, E, min(args.steps, 3), args.warmup, dev, stream,
                                       expert=not args.no_expert)
        line["surrogate_events"] = {
            "metric": "511keV events/s", "workload": E["desc"], "unit": "events/s",
            "value": r["value"], "e2e": r["e2e"], "plain_mc": r["mc_value"],
            "speedup_vs_plain_mc": r["value"] / r["mc_value"],
            "photopeak_shift": r["photopeak_shift"], "maps_vs_mc": r["maps"],
            "fallback_sites": r["stats"]["fallback_sites"], "sites": r["stats"]["sites"],
            "readout_face_expert": bool(r["experts"])}
    print(json.dumps(line), flush=True)
    eng.close()


def run_events_arm(args, rank, world, local_rank):
    """--workload events_csitl: events/s of the 511 keV event pipeline."""
    import torch
    import crysplight_b200 as cl
    if rank != 0 and args.impl == "reference":
        return
    E = events_workload(args.n_events or 50_000)
    if args.impl == "reference":
        base = events_cpu_baseline(E, args.cpu_seconds)
        for _ in range(args.warmup):
            pass
        line = {"impl": "reference", "metric": "511keV events/s", "value": base["value"],
                "unit": "events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 / base["value"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": E["name"], "desc": E["desc"]}, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "events/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    eng = cl.Engine(local_rank)
    r = run_events_bench(eng, E, args.steps, args.warmup, dev, stream, pid_base=0)
    dev_s, e2e_s = r["dev_s"], r["e2e_s"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, e2e_s = float(t[0]), float(t[1])
    if rank == 0:
        peaks = measured_peaks()
        n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
        ops = OPS_PER_STEP["point1m"]
        achieved = ops * r["photon_steps"] / dev_s
        peak = n_sm * 128 * peaks.get("sm_max_mhz", 1965.0) * 1e6
        line = {"metric": "511keV events/s", "value": world * E["n_events"] / dev_s,
                "unit": "events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_s * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": E["name"], "desc": E["desc"],
                           "photons_per_step": r["photons"], "deposits": r["deposits"],
                           "l2": "flushed between timed steps (256 MiB memset)",
                           "cuda_graph": True, "launch": r["launch"], "autotune_ms": r["tune_ms"]},
                "e2e": {"value": world * E["n_events"] / e2e_s, "unit": "events/s",
                        "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
                "gpu_launches": 3 * args.steps,
                "photon_steps_per_launch": r["photon_steps"],
                "roofline": {"bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9,
                             "unit": "Gop/s", "frac": achieved / peak, "traffic": None,
                             "ops_per_step": ops}}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = events_cpu_baseline(E, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    eng.close()


def run_surrogate_events_arm(args, rank, world, local_rank):
    """--workload events_bgo_surrogate: events/s of the surrogate + Monte Carlo
    fallback pipeline (500,000 BGO+ESR events), the plain CUDA Monte Carlo on the same events,
    and their agreement (photopeak, per-SiPM chi2)."""
    import torch
    import crysplight_b200 as cl
    E = surrogate_events_workload(args.n_events or 500_000)
    if args.impl == "reference":
        if rank != 0:
            return
        base = events_cpu_baseline(E, args.cpu_seconds)
        line = {"impl": "reference", "metric": "511keV events/s", "value": base["value"],
                "unit": "events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * E["n_events"] / base["value"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": E["name"], "desc": E["desc"]}, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "events/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    eng = cl.Engine(local_rank)
    clocks = ClockSampler(local_rank)
    clocks.start()
    r = run_surrogate_events_bench(eng, E, args.steps, args.warmup, dev, stream,
                                   wall_min_mm=args.wall_min_mm, expert=not args.no_expert)
    clk = clocks.stop()
    dev_s, e2e_s = r["dev_s"], E["n_events"] / r["e2e"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s, e2e_s = float(t[0]), float(t[1])
    if rank == 0:
        line = {"metric": "511keV events/s", "value": world * E["n_events"] / dev_s,
                "unit": "events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": dev_s * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+bf16", "data": "synthetic",
                "config": {"workload": E["name"], "desc": E["desc"], "deposits": r["deposits"],
                           "photons_per_step": r["photons"], "wall_min_mm": args.wall_min_mm,
                           "readout_face_expert": bool(r["experts"]),
                           "l2": "flushed between timed steps (256 MiB memset)"},
                "e2e": {"value": world * E["n_events"] / e2e_s, "unit": "events/s",
                        "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
                "gpu_launches": args.steps * r["launches"],
                "plain_mc": {"value": r["mc_value"], "unit": "events/s", "seconds": r["mc_s"],
                             "photon_steps": r["mc_photon_steps"]},
                "speedup_vs_plain_mc": r["value"] / r["mc_value"],
                "sites": r["stats"], "photopeak_surrogate": r["photopeak_surrogate"],
                "photopeak_mc": r["photopeak_mc"], "photopeak_shift": r["photopeak_shift"],
                "maps_vs_mc": r["maps"], "clocks": clk}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = events_cpu_baseline(E, args.cpu_seconds)
        print(json.dumps(line), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("cuda", "reference"), default="cuda")
    ap.add_argument("--workload", choices=("scan256", "point1m", "events_csitl",
                                           "events_bgo_surrogate"),
                    default="scan256")
    ap.add_argument("--events", type=int, default=10_000,
                    help="events in the secondary events/s measurement of the default run "
                         "(0 = skip)")
    ap.add_argument("--surrogate-training", type=int, default=1,
                    help="add the surrogate MLP's training throughput to the default line (0 = skip)")
    ap.add_argument("--surrogate-events", type=int, default=500_000,
                    help="events in the secondary surrogate-vs-Monte-Carlo measurement of the "
                         "default run (0 = skip)")
    ap.add_argument("--n-events", type=int, default=0,
                    help="events of --workload events_csitl (default 50000) or "
                         "events_bgo_surrogate (default 500000)")
    ap.add_argument("--wall-min-mm", type=float, default=1.0,
                    help="events_bgo_surrogate: sites closer than this to a wrapped face "
                         "go to the Monte Carlo")
    ap.add_argument("--no-expert", action="store_true",
                    help="events_bgo_surrogate: the whole-crystal ensemble only, without the "
                         "readout-face expert")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--points", type=int, default=256,
                    help="scan256: use only the first N points (profiling of a smaller case)")
    ap.add_argument("--photons-per-point", type=int, default=200_000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "events_bgo_surrogate":
        run_surrogate_events_arm(args, rank, world, local_rank)
        return
    if args.workload == "events_csitl":
        if world > 1 and args.impl == "cuda":
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            run_events_arm(args, rank, world, local_rank)
        finally:
            if world > 1 and args.impl == "cuda":
                import torch.distributed as dist
                dist.destroy_process_group()
        return
    W = workload(args.workload, args.points, args.photons_per_point)
    if args.impl == "reference":
        run_reference_arm(args, W, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_cuda_arm(args, W, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
