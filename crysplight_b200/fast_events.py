"""511 keV events from the learned light-response surrogate, with the plain
Monte Carlo as fallback.

The event pipeline of the reference (``run_events!``, src/events.jl:39-125)
transports every scintillation photon of every deposit.  Here each deposit
("site") is first shown to the surrogate ensemble (``LightSurrogate``: K MLPs
resident on the GPU, evaluated by the library's tcgen05 forward kernels); the
ensemble mean gives per SiPM the probability that one photon emitted at the
site is detected there, and the transit-time mean and spread of the detected
photons (the sites' inputs are scaled, and the depth warped, on the device by
``cl_surrogate_inputs``).  A site is sent to the Monte Carlo instead when the members disagree
(relative spread above ``spread_max``, default 2%), when it lies within
``wall_min_mm`` (default 1 mm) of a wrapped face, where the light response
changes fastest, or when its probabilities do not form a valid split.
Trusted sites are sampled by ``cl_run_events_surrogate_device``: the site's
Poisson photon count (drawn by the host gamma stage exactly as for the Monte
Carlo) is split over the SiPMs multinomially and each SiPM's first-hit time is
drawn as the minimum of its photons' emission delay plus transit time.  Both
kinds of sites feed the same per-event maps in one device call.

The surrogate is trained at PDE 1; the PDE of the run multiplies its
probabilities, which is exact because the reference detects a photon that
entered a SiPM by one last independent draw against the PDE
(src/transport.jl:161-185).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from .events import EventsResult, GammaMaterial, gamma_stage
from .params import COUNTER_NAMES, Box, OpticalParams, Readout, TimeBinning
from .surrogate import D_OUT, MLP, N_CELLS, LightSurrogate, first_pass_light, first_pass_optics
from .transport import stream_arg

SPREAD_MAX = 0.02
WALL_MIN_MM = 1.0


@dataclass
class SiteLight:
    """Per-site outputs of the ensemble (CUDA tensors)."""
    p: object          # (n, 64) float32, detection probability per photon (PDE applied)
    tmean: object      # (n, 64) float32 ns
    tsig: object       # (n, 64) float32 ns
    spread: object     # (n,) float32
    flag: object       # (n,) uint8: 1 spread, 2 near a wrapped face, 4 invalid


class _Resident:
    """One ensemble's networks and output scaling on the GPU."""

    def __init__(self, sur: LightSurrogate, device: int, dev, max_batch: int):
        import torch
        self.sur = sur
        self.nets = []
        for p in sur.members:
            net = MLP(device, max_batch=max_batch, seed=0)
            net.set_params(p)
            self.nets.append(net)
        self.y_mean = torch.from_numpy(np.ascontiguousarray(sur.y_mean, np.float32)).to(dev)
        self.y_std = torch.from_numpy(np.ascontiguousarray(sur.y_std, np.float32)).to(dev)
        z0, z1 = sur.depth_range()
        self.z0 = z0
        # the network's input box: x, y over the crystal, depth over its slab
        self.in_box = Box((float(sur.box_mm[0]), float(sur.box_mm[1]), z1 - z0))

    def close(self):
        for n in self.nets:
            n.close()
        self.nets = []


class SurrogateEvents:
    """A ``LightSurrogate`` resident on one GPU and the surrogate event
    generator built on it.  Not re-entrant.

    ``experts``: ensembles trained on a depth slab (``LightSurrogate.z_range``)
    of the same crystal, e.g. the last millimetres before the readout face,
    where the light of a site concentrates under one SiPM and one network for
    the whole crystal is least certain.  A site deeper than an expert's slab
    start plus ``expert_margin_mm`` takes that expert's outputs (spread and
    flags included) instead of the main ensemble's; the margin keeps the
    slab's edge, where its training data ends, out of use."""

    def __init__(self, surrogate: LightSurrogate, engine=None, device: int = 0,
                 max_batch: int = 65536, experts=(), expert_margin_mm: float = 1.0):
        import torch
        from .transport import Engine
        self.sur = surrogate
        self.device = device
        self.dev = torch.device("cuda", device)
        self.engine = engine or Engine(device)
        self.lib = _lib.load()
        self.box = Box(tuple(float(v) for v in surrogate.box_mm))
        self.main = _Resident(surrogate, device, self.dev, max_batch)
        self.experts = []
        for e in experts:
            if tuple(float(v) for v in e.box_mm) != tuple(float(v) for v in surrogate.box_mm):
                raise ValueError("an expert was trained for another crystal size")
            if e.z_range is None:
                raise ValueError("an expert needs a depth range (LightSurrogate.z_range)")
            self.experts.append(_Resident(e, device, self.dev, max_batch))
        self.expert_margin_mm = float(expert_margin_mm)

    @property
    def nets(self):
        return self.main.nets

    def _check_first_pass(self, op: OpticalParams, ro: Readout):
        """An ensemble trained on the light minus the first-pass term serves
        only the optics that term was computed for."""
        want = first_pass_optics(op, ro)
        for r in [self.main] + self.experts:
            fp = r.sur.first_pass
            if fp is not None and not np.array_equal(np.float32(fp), np.float32(want)):
                raise ValueError(f"the ensemble's first-pass term is for optics {fp}, the run has {want}")

    def close(self):
        for r in [self.main] + self.experts:
            r.close()

    def _light(self, ens: _Resident, xyz, ro: Readout, pde: float, spread_max: float,
               wall_min_mm: float, stream) -> SiteLight:
        """One ensemble on sites xyz ((n, 3) float32 CUDA tensor, mm)."""
        import torch
        n = int(xyz.shape[0])
        K = len(ens.nets)
        xyz = xyz.contiguous()
        xin = torch.empty((n, 3), dtype=torch.float32, device=self.dev)
        xs = xyz
        if ens.z0 != 0.0:
            xs = xyz - torch.tensor([0.0, 0.0, ens.z0], dtype=torch.float32, device=self.dev)
        rc = self.lib.cl_surrogate_inputs(C.c_void_p(xs.data_ptr()), n, C.byref(ens.in_box),
                                          float(ens.sur.z_warp), C.c_void_p(xin.data_ptr()),
                                          stream_arg(stream))
        if rc != 0:
            raise _lib.CudaTransportError(rc, "cl_surrogate_inputs failed")
        torch.cuda.synchronize(self.dev)         # the networks run on their own streams
        raw = torch.empty((K, n, D_OUT), dtype=torch.float32, device=self.dev)
        for k, net in enumerate(ens.nets):
            if n:
                net.forward_into(xin, raw[k])
        out = SiteLight(torch.empty((n, N_CELLS), dtype=torch.float32, device=self.dev),
                        torch.empty((n, N_CELLS), dtype=torch.float32, device=self.dev),
                        torch.empty((n, N_CELLS), dtype=torch.float32, device=self.dev),
                        torch.empty(n, dtype=torch.float32, device=self.dev),
                        torch.empty(n, dtype=torch.uint8, device=self.dev))
        P = C.c_void_p
        # an ensemble trained on the light minus the first-pass term gets it back here
        direct = None
        if ens.sur.first_pass is not None and n:
            direct = first_pass_light(xyz, self.box, ens.sur.first_pass, self.device, stream)
        rc = self.lib.cl_surrogate_combine_direct(
            P(raw.data_ptr()), K, n, P(ens.y_mean.data_ptr()), P(ens.y_std.data_ptr()),
            P(xyz.data_ptr()), P(direct.data_ptr()) if direct is not None else None, C.byref(self.box),
            C.byref(ro), float(pde), float(spread_max),
            float(wall_min_mm), P(out.p.data_ptr()), P(out.tmean.data_ptr()), P(out.tsig.data_ptr()),
            P(out.spread.data_ptr()), P(out.flag.data_ptr()), stream_arg(stream))
        if rc != 0:
            raise _lib.CudaTransportError(rc, "cl_surrogate_combine failed")
        return out

    def site_light(self, xyz, *, ro: Readout, pde: float, spread_max: float = SPREAD_MAX,
                   wall_min_mm: float = WALL_MIN_MM, stream=None) -> SiteLight:
        """Ensemble outputs for sites xyz ((n, 3) float32 CUDA tensor, mm),
        each site from the main ensemble or the expert whose slab holds it."""
        import torch
        out = self._light(self.main, xyz, ro, pde, spread_max, wall_min_mm, stream)
        for ens in self.experts:
            z0, z1 = ens.sur.depth_range()
            z = xyz[:, 2]
            idx = torch.nonzero((z >= z0 + self.expert_margin_mm) & (z <= z1)).flatten()
            if idx.numel() == 0:
                continue
            sub = self._light(ens, xyz.index_select(0, idx), ro, pde, spread_max, wall_min_mm, stream)
            torch.cuda.synchronize(self.dev)     # both combines ran on `stream`
            for name in ("p", "tmean", "tsig", "spread", "flag"):
                getattr(out, name).index_copy_(0, idx, getattr(sub, name))
        if self.experts:
            torch.cuda.synchronize(self.dev)
        return out

    def transport_sites(self, box: Box, op: OpticalParams, ro: Readout, tb: TimeBinning, *,
                        xyz, t0, photons, segment, n_segments: int, seed: int, tau_ns: float,
                        pid_offset: int = 0, max_bounces: int = 100_000,
                        spread_max: float = SPREAD_MAX, wall_min_mm: float = WALL_MIN_MM,
                        stream=None, light: Optional[SiteLight] = None):
        """Maps of ``n_segments`` events from their sites, all inputs CUDA
        tensors: xyz (n, 3) float32 mm, t0 (n,) float32 ns, photons (n,) int64,
        segment (n,) int32 non-decreasing.  ``light`` overrides the ensemble's
        site outputs.  Returns device tensors (maps int32 [n_seg*64], tmin
        float32, npe int32, counters int64[9], sampled int64[2]) and a dict of
        site statistics."""
        if (float(box.L[0]), float(box.L[1]), float(box.L[2])) != tuple(float(v) for v in self.sur.box_mm):
            raise ValueError("the surrogate was trained for another crystal size")
        ro = ro if isinstance(ro, Readout) else Readout(ro)
        if light is None:
            self._check_first_pass(op, ro)
            light = self.site_light(xyz, ro=ro, pde=float(op.pde), spread_max=spread_max,
                                    wall_min_mm=wall_min_mm, stream=stream)
        return sample_sites(self.engine, box, op, ro, tb, xyz=xyz, t0=t0, photons=photons,
                            segment=segment, n_segments=n_segments, seed=seed, tau_ns=tau_ns,
                            light=light, pid_offset=pid_offset, max_bounces=max_bounces, stream=stream)

    def run_events(self, box: Box, op: OpticalParams, ro, tb: TimeBinning, material: GammaMaterial,
                   yield_per_mev: float, *, n_events: int, seed: int, tau_ns: float,
                   e0_mev: float = 0.511, max_bounces: int = 100_000, nthreads: int = 0,
                   spread_max: float = SPREAD_MAX, wall_min_mm: float = WALL_MIN_MM,
                   gamma=None) -> EventsResult:
        """``run_events!`` (src/events.jl:39-125) with the surrogate for the
        trusted sites.  ``gamma`` may pass a precomputed host gamma stage."""
        import torch
        ro = ro if isinstance(ro, Readout) else Readout(ro)
        n = int(n_events)
        g = gamma if gamma is not None else gamma_stage(material, box, n_events=n, seed=seed,
                                                        yield_per_mev=yield_per_mev, e0_mev=e0_mev,
                                                        nthreads=nthreads)
        nx, ny = ro.grid.nx, ro.grid.ny
        out = EventsResult(g.edep.copy(), np.zeros(n, np.int32),
                           np.zeros((nx, ny, n), np.uint16, order="F"),
                           np.full((nx, ny, n), np.inf, np.float32, order="F"),
                           g.xyz1.copy(order="F"), g.e1.copy(), g.xyz2.copy(order="F"), g.e2.copy(),
                           g.er.copy(), g.int_type.copy(), g.n_int.copy())
        if g.dep_photons.size == 0:
            out.counters = {k: 0 for k in COUNTER_NAMES}
            return out
        dev = self.dev
        xyz = torch.from_numpy(np.ascontiguousarray(g.dep_xyz, np.float32)).to(dev)
        t0 = torch.from_numpy(np.ascontiguousarray(g.dep_t, np.float32)).to(dev)
        ph = torch.from_numpy(np.ascontiguousarray(g.dep_photons, np.int64)).to(dev)
        seg = torch.from_numpy(np.ascontiguousarray(g.dep_event, np.int32)).to(dev)
        (maps, tmin, npe, ctr, sampled), stats = self.transport_sites(
            box, op, ro, tb, xyz=xyz, t0=t0, photons=ph, segment=seg, n_segments=n, seed=seed,
            tau_ns=tau_ns, max_bounces=max_bounces, spread_max=spread_max, wall_min_mm=wall_min_mm)
        # the device maps are [event][cell], the memory order of the Fortran
        # (nx, ny, n) arrays: copy straight into them (UInt16 maps wrap as in Julia)
        torch.from_numpy(out.maps.reshape(-1, order="F").view(np.int16)).copy_(
            (maps & 0xFFFF).to(torch.int16))
        torch.from_numpy(out.tmin.reshape(-1, order="F")).copy_(tmin)
        torch.from_numpy(out.npe).copy_(npe)
        out.n_photons = g.n_photons
        out.counters = dict(zip(COUNTER_NAMES, (int(v) for v in ctr.cpu().numpy())))
        s = sampled.cpu().numpy()
        stats.update({"photons_sampled": int(s[0]), "detections_sampled": int(s[1])})
        out.surrogate_stats = stats
        return out


def sample_sites(engine, box: Box, op: OpticalParams, ro: Readout, tb: TimeBinning, *, xyz, t0, photons,
                 segment, n_segments: int, seed: int, tau_ns: float, light: SiteLight,
                 pid_offset: int = 0, max_bounces: int = 100_000, stream=None):
    """One ``cl_run_events_surrogate_device`` call: the flagged sites through
    the Monte Carlo, the others sampled from ``light`` (see
    ``SurrogateEvents.transport_sites`` for the arguments and results)."""
    import torch
    dev = xyz.device
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    if stream:
        torch.cuda.ExternalStream(stream, device=dev).synchronize()
    else:
        torch.cuda.synchronize(dev)
    flag_h = light.flag.cpu().numpy()          # the host picks the fallback sites
    fb = np.nonzero(flag_h)[0]
    n_sites = int(xyz.shape[0])
    if fb.size:
        fb_d = torch.from_numpy(fb).to(dev)
        sx, sy, sz = (xyz[fb_d, i].contiguous() for i in range(3))
        st = t0[fb_d].contiguous()
        cnt = photons[fb_d]
        off = torch.zeros(fb.size + 1, dtype=torch.int64, device=dev)
        torch.cumsum(cnt, 0, out=off[1:])
        seg = segment[fb_d].contiguous()
        n_mc = int(off[-1].item())
    else:
        sx = sy = sz = st = off = seg = None
        n_mc = 0
    maps = torch.empty(n_segments * N_CELLS, dtype=torch.int32, device=dev)
    tmin = torch.empty(n_segments * N_CELLS, dtype=torch.float32, device=dev)
    npe = torch.empty(n_segments, dtype=torch.int32, device=dev)
    ctr = torch.empty(9, dtype=torch.int64, device=dev)
    sampled = torch.empty(2, dtype=torch.int64, device=dev)
    P = C.c_void_p

    def ptr(t):
        return P(t.data_ptr()) if t is not None else None
    eng = engine
    rc = _lib.load().cl_run_events_surrogate_device(
        eng.handle, C.byref(box), C.byref(op), C.byref(ro), C.byref(tb),
        ptr(sx), ptr(sy), ptr(sz), ptr(st), ptr(off), ptr(seg), int(fb.size), n_mc,
        int(seed), int(pid_offset), float(np.float32(tau_ns)), int(max_bounces),
        ptr(light.p), ptr(light.tmean), ptr(light.tsig), ptr(light.flag), ptr(t0.contiguous()),
        ptr(photons.contiguous()), ptr(segment.contiguous()), n_sites, int(seed) & 0xFFFFFFFFFFFFFFFF,
        int(n_segments), ptr(maps), ptr(tmin), ptr(npe), ptr(ctr), ptr(sampled),
        stream_arg(stream))
    eng._check(rc)
    # the site statistics are gathered while the transport runs (torch's own
    # stream; `photons` is only read by both)
    wall = torch.from_numpy((flag_h & 2) != 0).to(dev)
    stats = {"sites": n_sites, "fallback_sites": int(fb.size), "photons_mc": n_mc,
             "photons_total": int(photons.sum().item()),
             "photons_wall": int(photons[wall].sum().item()) if bool(wall.any()) else 0,
             "flag_spread": int(np.count_nonzero(flag_h & 1)),
             "flag_wall": int(np.count_nonzero(flag_h & 2)),
             "flag_invalid": int(np.count_nonzero(flag_h & 4))}
    eng.sync(stream)
    return (maps, tmin, npe, ctr, sampled), stats


# ---------------------------------------------------------------------------
# Comparison against the plain Monte Carlo on the same events
# ---------------------------------------------------------------------------
def photopeak(npe: np.ndarray, edep_kev: np.ndarray, e0_kev: float = 511.0, tol_kev: float = 1.0) -> dict:
    """Summed-light photopeak of the full-absorption events (deposited energy
    within tol of e0): mean, standard deviation and FWHM (2.3548 sigma) of npe."""
    sel = np.abs(np.asarray(edep_kev, np.float64) - e0_kev) <= tol_kev
    v = np.asarray(npe, np.float64)[sel]
    if v.size < 2:
        return {"events": int(v.size), "mean": float("nan"), "sigma": float("nan"), "fwhm_rel": float("nan")}
    mu, sd = float(v.mean()), float(v.std(ddof=1))
    return {"events": int(v.size), "mean": mu, "sigma": sd, "fwhm_rel": 2.3548 * sd / mu,
            "mean_err": sd / np.sqrt(v.size)}


def compare_maps(maps_a: np.ndarray, maps_b: np.ndarray) -> dict:
    """Per-SiPM agreement of two event samples over the same events: the
    relative difference of each SiPM's summed counts (mean and max over
    SiPMs), and per SiPM chi2 / ndf = mean over events of (a - b)^2 / (a + b)
    (about 1 when both are independent draws of the same distribution)."""
    a = np.asarray(maps_a, np.float64).reshape(-1, maps_a.shape[-1])
    b = np.asarray(maps_b, np.float64).reshape(-1, maps_b.shape[-1])
    sa, sb = a.sum(1), b.sum(1)
    rel = np.abs(sa - sb) / np.maximum(sb, 1.0)
    den = a + b
    ok = den > 0
    chi = np.where(ok, (a - b) ** 2 / np.where(ok, den, 1.0), 0.0)
    chi_ndf = chi.sum(1) / np.maximum(ok.sum(1), 1)
    return {"rel_mean": float(rel.mean()), "rel_max": float(rel.max()),
            "chi2_ndf_mean": float(chi_ndf.mean()), "chi2_ndf_max": float(chi_ndf.max())}
