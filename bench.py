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
# DRAM bytes (read + write) per photon-step of the transport kernel, from one
# ncu capture of each workload at a reduced size (scan: 20,000 photons per
# point, 3.01 GB for 494.8M photon-steps; point source: the whole 10^6-photon
# launch, 143 MB for 12.33M photon-steps, mostly the table's first touches),
# scaled to a full launch by its photon-steps.  Almost all of it is L2 misses of the 64 MB log table (about 2
# bytes per photon-step and lookup), which grow in proportion to the steps;
# the sources, offsets and maps are 0.24 MB.
TRAFFIC_PER_STEP = {"scan256": (3.003462e9 + 7.173888e6) / 494_804_727,
                    "point1m": (139.735552e6 + 3.632384e6) / 12_332_791}
# Warp instructions the transport kernel issues per photon-step (smsp__inst_executed
# of the same ncu captures: 15.42 G for 494.8M photon-steps on the scan, 0.80 G
# for 12.33M on the point source); with the live steps/s this gives the
# kernel's issue rate against the SMs' issue slots.
WARP_INST_PER_STEP = {"scan256": 15_422_450_065 / 494_804_727, "point1m": 804_971_827 / 12_332_791}


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


def run_events_bench(eng, E, steps: int, warmup: int, dev, stream, pid_base: int = 0,
                     tune_events: int = 0):
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
    if tune_events and tune_events < E["n_events"]:
        # the launch shape is timed on the first tune_events events (same photons and streams)
        k = int(np.searchsorted(g.dep_event, tune_events, side="left"))
        ev_t = DeviceEvents(eng, E["box"], E["op"], E["ro"], E["tb"], xyz=T(g.dep_xyz[:k]),
                            t0=T(g.dep_t[:k]), photons=T(g.dep_photons[:k]),
                            segment=T(g.dep_event[:k]), n_segments=tune_events, seed=E["seed"],
                            tau_ns=E["tau"], pid_offset=pid_base)
        best, tune_times = autotune(eng, ev_t.step, stream=stream, repeats=2)
        del ev_t
    else:
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
    e2e_steps = min(steps, 5)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run_events(E["box"], E["op"], E["ro"], E["tb"], E["mat"], E["yield_"],
                   n_events=E["n_events"], seed=E["seed"], tau_ns=E["tau"], engine=eng)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
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
            "peak_source": measured_peaks().get("source", "measured"),
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
                               expert: bool = True, expert_files=None):
    """events/s of the surrogate + fallback pipeline with the deposits in HBM
    (value), the plain Monte Carlo on the same deposits, their agreement, and
    the whole public call SurrogateEvents.run_events (e2e)."""
    import torch
    from crysplight_b200.events import gamma_stage
    from crysplight_b200.fast_events import SurrogateEvents, compare_maps, photopeak
    from crysplight_b200.surrogate import LightSurrogate
    sur = LightSurrogate.load(SURROGATE_BGO)
    files = expert_files if expert_files else ([SURROGATE_BGO_FACE] if os.path.exists(SURROGATE_BGO_FACE) else [])
    experts = [LightSurrogate.load(f) for f in files] if expert else []
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
    tcmp = compare_first_times(tmin.cpu().numpy().reshape(n_seg, 64), s_maps,
                               m_tmin.cpu().numpy().reshape(n_seg, 64), mm)
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
    # the rule's ceiling: with the surrogate free, only the sites within the
    # wall margin would still go through the Monte Carlo
    ceiling = stats["photons_total"] / max(stats["photons_wall"], 1)
    return dict(value=n_seg / dev_s, e2e=n_seg / e2e_s, dev_s=dev_s, mc_value=n_seg / mc_s,
                ceiling_speedup=ceiling,
                mc_s=mc_s, mc_photon_steps=mc_steps, photons=int(off[-1]), deposits=nd,
                members=len(sur.members), experts=len(experts), launches=launches,
                stats=stats, photopeak_surrogate=pk_s, photopeak_mc=pk_m,
                photopeak_shift=(pk_s["mean"] - pk_m["mean"]) / pk_m["mean"], maps=cmp, first_times=tcmp,
                h2d=int(12 * nd + 4 * nd + 8 * nd + 4 * nd), d2h=int(2 * 4 * 64 * n_seg + 4 * n_seg + 72 + 16 + nd))


def compare_first_times(t_a, maps_a, t_b, maps_b) -> dict:
    """Per-SiPM first-hit times of two event samples over the same events: for
    each SiPM, the mean over the events where both have hits; the mean and the
    largest absolute difference of those means over the SiPMs (ns), the
    largest in units of its standard error, and the overall mean time."""
    both = (maps_a > 0) & (maps_b > 0) & np.isfinite(t_a) & np.isfinite(t_b)
    diffs, zs = [], []
    for c in range(t_a.shape[1]):
        m = both[:, c]
        if m.sum() < 20:
            continue
        d = t_a[m, c].astype(np.float64) - t_b[m, c]
        diffs.append(d.mean())
        zs.append(abs(d.mean()) / max(d.std(ddof=1) / np.sqrt(m.sum()), 1e-12))
    diffs = np.abs(np.array(diffs))
    return {"sipms": int(diffs.size), "mean_abs_diff_ns": float(diffs.mean()) if diffs.size else None,
            "max_abs_diff_ns": float(diffs.max()) if diffs.size else None,
            "max_z": float(max(zs)) if zs else None,
            "mean_first_time_ns": float(np.mean(t_b[both])) if both.any() else None}


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
    """MEASURED_PEAKS.json (measured on this pool's B200s), else the earlier
    measurement the profiling notes give as the fallback (marked)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        d.setdefault("source", "measured")
        return d
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "sm_max_mhz": 1965.0, "source": "fallback"}


# ------------------------------------------------------------------------------------
# reference arm / CPU baseline: the oracle on the host cores
# ------------------------------------------------------------------------------------
def cpu_run(W, per_point: int) -> tuple[float, int, int]:
    """The oracle on all host threads over every point of the workload with
    ``per_point`` photons each: (seconds, photons, photon-steps)."""
    from oracle import oracle
    pts = W["points"]
    n_points = pts.shape[0]
    t0 = time.perf_counter()
    if W["name"] == "scan256":
        _, steps = oracle.run_segments(W["box"], W["op"], W["ro"], W["tb"], sources=pts,
                                       photons_per_source=[per_point] * n_points,
                                       segment_of_source=range(n_points), n_segments=n_points,
                                       seed=W["seed"], tau_ns=W["tau"], nthreads=os.cpu_count(),
                                       return_steps=True)
    else:
        _, steps = oracle.run_photons_ka(W["box"], W["op"], W["ro"], W["tb"], n_photons=per_point,
                                         seed=W["seed"], pos=tuple(pts[0]), tau_ns=W["tau"],
                                         nthreads=os.cpu_count(), return_steps=True)
    dt = time.perf_counter() - t0
    return dt, n_points * per_point, int(steps)


def cpu_sample_size(W, target_s: float) -> int:
    """Photons per point of a sample over all the workload's points (the same
    points, optics and seed) that takes about target_s on the host."""
    probe = 2_000 if W["name"] == "scan256" else 20_000
    dt, _, _ = cpu_run(W, probe)
    per = int(probe * target_s / max(dt, 1e-3))
    return int(max(probe, min(W["per_point"], per)))


def cpu_sample_desc(W, per: int, dt: float) -> str:
    pts = W["points"].shape[0]
    return (f"all {pts} point(s) of the {W['name']} workload x {per} photons "
            f"({dt:.1f} s on {os.cpu_count()} threads)")


def cpu_baseline(W, target_s: float) -> dict:
    per = cpu_sample_size(W, target_s)
    dt, n, steps = cpu_run(W, per)
    reps = 1
    while dt < 0.5 * target_s:          # the whole workload is shorter than the target: repeat it
        d2, n2, s2 = cpu_run(W, per)
        dt, n, steps, reps = dt + d2, n + n2, steps + s2, reps + 1
    sample = cpu_sample_desc(W, per, dt) + (f", {reps} runs" if reps > 1 else "")
    return {"value": n / dt, "unit": "photons/s", "cores": os.cpu_count(), "kind": "port",
            "photon_steps_per_s": steps / dt, "sample": sample}


def workload_config(W) -> dict:
    """The workload the line is quoted on (the same dict in both arms)."""
    return {"workload": W["name"], "desc": W["desc"], "photons_per_step": W["n"]}


def run_reference_arm(args, W, rank, world):
    if rank != 0:
        return
    per = cpu_sample_size(W, args.cpu_seconds)
    for _ in range(args.warmup):
        cpu_run(W, per)
    times, tot_n, tot_steps = [], 0, 0
    for _ in range(args.steps):
        dt, n, st = cpu_run(W, per)
        times.append(dt)
        tot_n += n
        tot_steps += st
    value = tot_n / sum(times)
    sample = cpu_sample_desc(W, per, sum(times) / len(times)) + \
        " per step (C restatement of the reference CPU transport)"
    line = {
        "impl": "reference", "metric": "photons/s", "value": value, "unit": "photons/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(W),
        "photon_steps_per_s": tot_steps / sum(times),
        "cpu_baseline": {"value": value, "unit": "photons/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------
# CUDA arm
# ------------------------------------------------------------------------------------
def measure_photons(eng, W, steps: int, warmup: int, dev, stream, pid_base: int = 0,
                    clocks: bool = True) -> dict:
    """photons/s of one workload: ``value`` with the inputs resident in HBM
    (device entry point, CUDA events on the launch stream, L2 flushed between
    steps) and ``e2e`` through the host-buffer C-ABI call (pinned host inputs
    copied in, maps / times / counters copied out), timed by the host clock."""
    import torch
    nx = ny = 8
    pts = W["points"]
    npts = pts.shape[0]
    if W["name"] == "scan256":
        off = np.zeros(npts + 1, np.int64)
        off[1:] = np.cumsum(np.full(npts, W["per_point"], np.int64))
        seg = np.arange(npts, dtype=np.int32)
        d_sx, d_sy, d_sz = (torch.from_numpy(np.ascontiguousarray(pts[:, i])).to(dev) for i in range(3))
        d_off = torch.from_numpy(off).to(dev)
        d_seg = torch.from_numpy(seg).to(dev)
        d_maps = torch.empty(nx * ny * npts, dtype=torch.int32, device=dev)
        d_tmin = torch.empty(nx * ny * npts, dtype=torch.float32, device=dev)
        d_npe = torch.empty(npts, dtype=torch.int32, device=dev)
        d_ctr = torch.empty(9, dtype=torch.int64, device=dev)
        sptr = stream.cuda_stream

        def device_step():
            eng.run_segments_device(
                W["box"], W["op"], W["ro"], W["tb"], sx=d_sx.data_ptr(), sy=d_sy.data_ptr(),
                sz=d_sz.data_ptr(), st=None, src_offsets=d_off.data_ptr(),
                src_segment=d_seg.data_ptr(), n_src=npts, n_segments=npts, n_photons=W["n"],
                seed=W["seed"], pid_offset=pid_base, tau_ns=W["tau"], maps=d_maps.data_ptr(),
                tmin=d_tmin.data_ptr(), npe=d_npe.data_ptr(), counters=d_ctr.data_ptr(),
                stream=sptr)

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
        in_bytes = 3 * 4 * npts + 8 * (npts + 1) + 4 * npts
        out_bytes = 2 * 4 * nx * ny * npts + 4 * npts + 72
        launches = 3
    else:
        d_p = [torch.from_numpy(np.ascontiguousarray(pts[:, i])).to(dev) for i in range(3)]
        nb = W["tb"].nbins + 1
        d_counts = torch.empty(nx * ny * nb, dtype=torch.int32, device=dev)
        d_first = torch.empty(nx * ny, dtype=torch.float32, device=dev)
        d_ctr = torch.empty(9, dtype=torch.int64, device=dev)
        sptr = stream.cuda_stream

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
        in_bytes = 3 * 4
        out_bytes = 4 * nx * ny * nb + 4 * nx * ny + 72
        launches = 2

    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(warmup):
        device_step()
    eng.sync(sptr)
    host_step()

    clk = ClockSampler(dev.index or 0) if clocks else None
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    torch.cuda.synchronize(dev)
    if clk:
        clk.start()
    t_wall0 = time.perf_counter()
    for i in range(steps):
        flush.zero_()                       # evict L2 between timed steps
        starts[i].record(stream)
        device_step()
        stops[i].record(stream)
    eng.sync(sptr)
    torch.cuda.synchronize(dev)
    t_wall = time.perf_counter() - t_wall0
    clk_rec = clk.stop() if clk else None
    tot_ms = sum(s.elapsed_time(e) for s, e in zip(starts, stops))
    steps_per_launch = eng.last_steps

    torch.cuda.synchronize(dev)
    e2e_t0 = time.perf_counter()
    for _ in range(steps):
        host_step()
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - e2e_t0
    return dict(tot_ms=tot_ms, e2e_s=e2e_s, steps_per_launch=steps_per_launch, h2d=h2d, d2h=d2h,
                in_bytes=in_bytes, out_bytes=out_bytes, launches=launches, clocks=clk_rec,
                wall_s=t_wall)


def roofline(W, steps_per_launch: int, launch_s: float, in_bytes: int, out_bytes: int, n_sm: int) -> dict:
    """The transport kernel against the SMs' lane-op ceiling (its bound), its
    issue rate against the issue slots, and its DRAM traffic (the L2 misses of
    the 64 MB log table dominate it) against HBM."""
    peaks = measured_peaks()
    sm_mhz = peaks.get("sm_max_mhz", 1965.0)
    ops_step = OPS_PER_STEP[W["name"]]
    achieved = ops_step * steps_per_launch / launch_s
    peak = n_sm * 128 * sm_mhz * 1e6
    tps = TRAFFIC_PER_STEP.get(W["name"])
    traffic = tps * steps_per_launch if tps else None
    hbm_peak = peaks.get("hbm_gbs", 6553.3)
    dram = traffic if traffic is not None else float(in_bytes + out_bytes)
    return {
        "bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gop/s",
        "frac": achieved / peak, "traffic": traffic, "ops_per_step": ops_step,
        "peak_source": peaks.get("source", "measured"),
        "note": ("reference Float32/int ops per photon-step x steps / launch time, against "
                 "one op per lane per clock (SMs x 128 lanes x max SM clock of measured)"),
        "hbm": {"achieved": dram / launch_s / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": dram / launch_s / 1e9 / hbm_peak, "dram_bytes": dram,
                "algorithmic_bytes": in_bytes + out_bytes,
                "note": ("DRAM bytes per launch (ncu dram__bytes read+write per photon-step x "
                         "steps: L2 misses of the log table) over the launch time; the "
                         "algorithmic bytes are the sources, offsets, maps, times and counters")},
        "issue_slots": issue_slots(W["name"], steps_per_launch / launch_s, n_sm, sm_mhz),
    }


def run_cuda_arm(args, W, rank, world, local_rank):
    import torch
    import crysplight_b200 as cl
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1 or args.sharded:
        run_sharded_arm(args, W, rank, world, local_rank)
        return
    eng = cl.Engine(local_rank)
    stream = torch.cuda.Stream(dev)  # explicit stream: the library launches on it
    torch.cuda.set_stream(stream)
    r = measure_photons(eng, W, args.steps, args.warmup, dev, stream)
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    launch_s = r["tot_ms"] * 1e-3 / args.steps
    n_total = W["n"] * args.steps
    line = {
        "metric": "photons/s", "value": n_total / (r["tot_ms"] * 1e-3), "unit": "photons/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": r["tot_ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(W),
        "l2": "flushed between timed steps (256 MiB memset)", "parallelism": "1 GPU",
        "e2e": {"value": n_total / r["e2e_s"], "unit": "photons/s", "h2d_bytes_per_step": r["h2d"],
                "d2h_bytes_per_step": r["d2h"]},
        "gpu_launches": r["launches"] * args.steps,
        "photon_steps_per_launch": r["steps_per_launch"],
        "photon_steps_per_s": r["steps_per_launch"] / launch_s,
        "roofline": roofline(W, r["steps_per_launch"], launch_s, r["in_bytes"], r["out_bytes"], n_sm),
        "clocks": r["clocks"],
        "wall_s_timed": r["wall_s"],
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(W, args.cpu_seconds)
    if W["name"] == "scan256" and args.point1m:
        # config 1 at its stated size: 10^6 CsI(Tl)+Teflon photons from the centre
        P = workload("point1m")
        # a 1.2 ms launch: 25x the steps, so the clock sampler sees the timed region
        psteps = 25 * args.steps
        rp = measure_photons(eng, P, psteps, args.warmup, dev, stream)
        ls = rp["tot_ms"] * 1e-3 / psteps
        obj = {"metric": "photons/s", "workload": P["desc"], "unit": "photons/s", "steps": psteps,
               "value": P["n"] / ls, "e2e": {"value": P["n"] * psteps / rp["e2e_s"],
                                             "unit": "photons/s", "h2d_bytes_per_step": rp["h2d"],
                                             "d2h_bytes_per_step": rp["d2h"]},
               "ms_per_step": ls * 1e3, "photon_steps_per_launch": rp["steps_per_launch"],
               "photon_steps_per_s": rp["steps_per_launch"] / ls,
               "roofline": roofline(P, rp["steps_per_launch"], ls, rp["in_bytes"], rp["out_bytes"], n_sm),
               "clocks": rp["clocks"]}
        if not args.no_cpu_baseline:
            obj["cpu_baseline"] = cpu_baseline(P, args.cpu_seconds)
        line["point1m"] = obj
    if args.events > 0:
        # 511 keV events/s of the event pipeline (runs/gammas_csitl_50k.toml: 50,000 events)
        E = events_workload(args.events)
        r = run_events_bench(eng, E, args.steps, args.warmup, dev, stream,
                             tune_events=args.tune_events)
        obj = {"metric": "511keV events/s", "workload": E["desc"],
               "value": r["value"], "e2e": r["e2e"], "unit": "events/s",
               "photons_per_event": r["photons"] / E["n_events"],
               "photon_steps_per_s": r["photon_steps"] / r["dev_s"],
               "launch": r["launch"], "cuda_graph": True}
        if not args.no_cpu_baseline:
            obj["cpu_baseline"] = events_cpu_baseline(E, args.cpu_seconds)
        line["events"] = obj
    if args.surrogate_training:
        line["surrogate_training"] = surrogate_training_bench(dev)
    if args.surrogate_events > 0 and os.path.exists(SURROGATE_BGO):
        # secondary metric: 500,000 BGO+ESR events, surrogate + Monte Carlo fallback vs
        # the plain Monte Carlo
        E = surrogate_events_workload(args.surrogate_events)
        r = run_surrogate_events_bench(eng, E, min(args.steps, 3), args.warmup, dev, stream,
                                       expert=not args.no_expert, expert_files=args.experts)
        line["surrogate_events"] = {
            "metric": "511keV events/s", "workload": E["desc"], "unit": "events/s",
            "value": r["value"], "e2e": r["e2e"], "plain_mc": r["mc_value"],
            "speedup_vs_plain_mc": r["value"] / r["mc_value"],
            "ceiling_speedup": r["ceiling_speedup"],
            "photopeak_shift": r["photopeak_shift"], "maps_vs_mc": r["maps"],
            "first_times_vs_mc": r["first_times"],
            "fallback_sites": r["stats"]["fallback_sites"], "sites": r["stats"]["sites"],
            "readout_face_expert": bool(r["experts"])}
    print(json.dumps(line), flush=True)
    eng.close()


def run_sharded_arm(args, W, rank, world, local_rank):
    """N GPUs, one process each, on the product's multi-GPU path: one job of
    N copies of the workload's points (N x 256 segments, photon ids numbered
    over the whole job), split by whole segments over the ranks
    (sharding.ShardedSegments: each rank transports its share from HBM, then
    NCCL all_gather of every rank's maps / times / npe and all_reduce of the
    counters); the time of a step is the max over ranks of transport + gather.
    e2e: the same job through sharding.run_segments_sharded with host buffers."""
    import torch
    import torch.distributed as dist
    import crysplight_b200 as cl
    from crysplight_b200.sharding import ShardedSegments, run_segments_sharded
    if W["name"] != "scan256":
        raise SystemExit("--gpus N > 1 runs the scan256 workload")
    dev = torch.device("cuda", local_rank)
    eng = cl.Engine(local_rank)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    pts = np.tile(W["points"], (world, 1))
    nseg = pts.shape[0]
    cnt = np.full(nseg, W["per_point"], np.int64)
    seg = np.arange(nseg, dtype=np.int64)
    job = ShardedSegments(eng, W["box"], W["op"], W["ro"], W["tb"], sources=pts, photons_per_source=cnt,
                          segment_of_source=seg, n_segments=nseg, seed=W["seed"], tau_ns=W["tau"])
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        job.step()
    job.sync()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    torch.cuda.synchronize(dev)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        job.step()
        stops[i].record(stream)
    job.sync()
    torch.cuda.synchronize(dev)
    dist.barrier()
    clk = clocks.stop()
    tot_ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops))
    steps_local = eng.last_steps
    # end to end: host buffers through run_segments_sharded (copies, gather via NCCL)
    runner = lambda **kw: eng.run_segments(W["box"], W["op"], W["ro"], W["tb"], seed=W["seed"],
                                           tau_ns=W["tau"], **kw)
    run_segments_sharded(runner, sources=pts, photons_per_source=cnt, segment_of_source=seg,
                         n_segments=nseg)
    torch.cuda.synchronize(dev)
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        run_segments_sharded(runner, sources=pts, photons_per_source=cnt, segment_of_source=seg,
                             n_segments=nseg)
    torch.cuda.synchronize(dev)
    dist.barrier()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([tot_ms, e2e_s, float(steps_local)], dtype=torch.float64, device=dev)
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    sm = t.clone()
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    job = None
    if rank == 0:
        tot_ms, e2e_s = float(mx[0]), float(mx[1])
        n_total = int(cnt.sum()) * args.steps
        launch_s = tot_ms * 1e-3 / args.steps
        line = {
            "metric": "photons/s", "value": n_total / (tot_ms * 1e-3), "unit": "photons/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": tot_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(W),
            "job": f"{world} x {W['points'].shape[0]} points x {W['per_point']} photons, "
                   "whole-segment shards, NCCL all_gather of the maps",
            "l2": "flushed between timed steps (256 MiB memset)",
            "parallelism": f"segment shards x{world} (sharding.ShardedSegments)",
            "e2e": {"value": n_total / e2e_s, "unit": "photons/s",
                    "h2d_bytes_per_step": int(3 * 4 * nseg + 8 * (nseg + 1) + 4 * nseg),
                    "d2h_bytes_per_step": int(2 * 4 * 64 * nseg + 4 * nseg + 72)},
            "gpu_launches": 3 * args.steps,
            "photon_steps_per_s": float(sm[2]) / launch_s,
            "clocks": clk,
        }
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
    r = run_events_bench(eng, E, args.steps, args.warmup, dev, stream, pid_base=0,
                         tune_events=args.tune_events)
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
                                   wall_min_mm=args.wall_min_mm, expert=not args.no_expert,
                                   expert_files=args.experts)
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
                "maps_vs_mc": r["maps"], "first_times_vs_mc": r["first_times"], "clocks": clk}
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
                                           "events_bgo_surrogate", "surrogate_training"),
                    default="scan256")
    ap.add_argument("--events", type=int, default=50_000,
                    help="events in the secondary events/s measurement of the default run "
                         "(runs/gammas_csitl_50k.toml: 50,000; 0 = skip)")
    ap.add_argument("--point1m", type=int, default=1,
                    help="add the 10^6-photon CsI(Tl)+Teflon point source to the default line "
                         "(0 = skip)")
    ap.add_argument("--tune-events", type=int, default=5_000,
                    help="events of the sample the launch-shape autotuner times")
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
    ap.add_argument("--experts", nargs="*", default=None,
                    help="events_bgo_surrogate: depth-slab expert ensembles (.npz), applied in "
                         "order (default: the shipped readout-face expert)")
    ap.add_argument("--sharded", action="store_true",
                    help="scan256: the multi-GPU path (sharding.ShardedSegments with NCCL) even on "
                         "one rank (it is the default for more than one rank)")
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
    if args.workload == "surrogate_training":
        # the training leg alone (its line is also part of the default run)
        if rank != 0:
            return
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the surrogate has no counterpart "
                              "in the reference"}))
            return
        import torch
        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        print(json.dumps(surrogate_training_bench(dev, steps=args.steps, warmup=args.warmup)))
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
    distributed = world > 1 or args.sharded
    if distributed:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        os.environ.setdefault("RANK", str(rank))
        os.environ.setdefault("WORLD_SIZE", str(world))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_cuda_arm(args, W, rank, world, local_rank)
    finally:
        if distributed:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
