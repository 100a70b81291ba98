"""Splitting one transport over several GPUs (one process per GPU).

Photons are independent and every photon's Philox stream is keyed by its
global id (src/philox.jl:43, pid_offset of src/kernel.jl:317), so any
partition of the photon range reproduces the single-GPU result exactly; the
only exchange is one reduction of the small output maps at the end:

  * point sources (``run_photons_ka!``): rank r transports a contiguous range
    of photon ids; the count histograms and counters are summed and the
    first-hit times reduced by min (``reduce_accumulator``).  With several
    source positions the reference assigns photon i (within a call) to
    position i mod npos, so range starts are kept on multiples of npos;
  * events / scan points (``run_segments``): rank r owns a contiguous range of
    whole segments, chosen to balance photons, with pid_offset = photons
    before it; the per-segment maps are concatenated (``gather_segments``).

The collectives go through ``torch.distributed`` (NCCL between GPUs, gloo on
the host); ``runner`` callables do the per-rank transport, so the same logic
runs with the CUDA engine or, in tests, on the CPU.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np

from .params import Accumulator


def photon_range(n_photons: int, rank: int, world: int, align: int = 1) -> tuple[int, int]:
    """(first photon index, count) of ``rank``'s share of ``n_photons``:
    contiguous, balanced, every start a multiple of ``align``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    align = max(1, int(align))
    units = -(-int(n_photons) // align)             # ceil
    lo = (units * rank // world) * align
    hi = min(int(n_photons), (units * (rank + 1) // world) * align)
    return lo, max(0, hi - lo)


def segment_range(photons_per_segment: Sequence[int], rank: int, world: int) -> tuple[int, int, int]:
    """(first segment, end segment, photons before the first) of ``rank``'s
    contiguous share of whole segments, balanced by photon count."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    c = np.zeros(len(photons_per_segment) + 1, np.int64)
    np.cumsum(np.asarray(photons_per_segment, np.int64), out=c[1:])
    total = int(c[-1])
    # segment boundaries nearest to the equal-photon split points
    cut = []
    for k in range(world + 1):
        target = total * k / world
        i = int(np.searchsorted(c, target, side="left"))
        if i > 0 and (i >= c.size or target - c[i - 1] <= c[i] - target):
            i -= 1
        cut.append(i)
    cut[0], cut[-1] = 0, len(photons_per_segment)
    for k in range(1, world + 1):
        cut[k] = max(cut[k], cut[k - 1])
    lo, hi = cut[rank], cut[rank + 1]
    return lo, hi, int(c[lo])


def check_segments(photons_per_source, segment_of_source, n_segments: int):
    """Validate a segmented job as cl_run_segments does (src/events.jl:70,88
    numbers photons event-major, so the photons before a range of whole
    segments are the photons of the sources before it only when segment ids
    never decrease along the sources): returns (counts int64, segment int64)
    or raises ValueError.  Every rank checks the same arrays, so all ranks
    raise before any collective."""
    cnt = np.asarray(photons_per_source, np.int64).reshape(-1)
    seg = np.asarray(segment_of_source, np.int64).reshape(-1)
    if cnt.shape != seg.shape:
        raise ValueError("photons_per_source and segment_of_source differ in length")
    if int(n_segments) < 1:
        raise ValueError("need n_segments >= 1")
    if cnt.size and (cnt.min() < 0):
        raise ValueError("photons_per_source must be >= 0")
    if seg.size and (seg.min() < 0 or seg.max() >= int(n_segments)):
        raise ValueError("segment id out of range")
    if seg.size > 1 and np.any(np.diff(seg) < 0):
        raise ValueError("segment ids must be non-decreasing along the sources "
                         "(photon ids are numbered segment-major)")
    return cnt, seg


def shard_segments(photons_per_source, segment_of_source, n_segments: int, rank: int, world: int):
    """Rank ``rank``'s share of a segmented job: (first segment, end segment,
    first source, end source, photons before the first source).  The sources
    of segments [lo, hi) are the contiguous range [s0, s1) because segment ids
    are non-decreasing (checked)."""
    cnt, seg = check_segments(photons_per_source, segment_of_source, n_segments)
    per_seg = np.bincount(seg, weights=cnt, minlength=int(n_segments)).astype(np.int64)
    lo, hi, _ = segment_range(per_seg, rank, world)
    s0 = int(np.searchsorted(seg, lo, side="left"))
    s1 = int(np.searchsorted(seg, hi, side="left"))
    return lo, hi, s0, s1, int(cnt[:s0].sum())


def reduce_accumulator(acc: Accumulator, group=None) -> Accumulator:
    """All-reduce a per-rank Accumulator in place: counts and counters summed,
    first-hit times by min (src/transport.jl:82-91, ``merge!``)."""
    import torch
    import torch.distributed as dist
    from .params import COUNTER_NAMES
    dev = _collective_device(group)
    counts = torch.from_numpy(np.ascontiguousarray(acc.counts.ravel(order="F")).astype(np.int64)).to(dev)
    first = torch.from_numpy(np.ascontiguousarray(acc.first_ns.ravel(order="F"))).to(dev)
    ctr = torch.tensor([int(getattr(acc, n)) for n in COUNTER_NAMES], dtype=torch.int64, device=dev)
    dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(first, op=dist.ReduceOp.MIN, group=group)
    dist.all_reduce(ctr, op=dist.ReduceOp.SUM, group=group)
    acc.counts[...] = counts.cpu().numpy().astype(acc.counts.dtype).reshape(acc.counts.shape, order="F")
    acc.first_ns[...] = first.cpu().numpy().reshape(acc.first_ns.shape, order="F")
    for n, v in zip(COUNTER_NAMES, ctr.cpu().tolist()):
        setattr(acc, n, int(v))
    return acc


def gather_segments(arrays: Sequence[np.ndarray], n_local: int, group=None) -> list[np.ndarray]:
    """Concatenate, in rank order along the last (segment) axis, per-rank
    arrays holding ``n_local`` segments each (Fortran-ordered (..., n_local)).
    Every rank receives the full arrays."""
    import torch
    import torch.distributed as dist
    dev = _collective_device(group)
    world = dist.get_world_size(group)
    sizes = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([n_local], dtype=torch.int64, device=dev), group=group)
    sizes = [int(t.item()) for t in sizes]
    n_max = max(sizes) if sizes else 0
    out = []
    for a in arrays:
        a = np.asarray(a)
        lead = a.shape[:-1]
        per = int(np.prod(lead)) if lead else 1
        flat = np.zeros(per * n_max, dtype=a.dtype)
        flat[:per * n_local] = a.ravel(order="F")
        t = torch.from_numpy(flat.view(np.uint8)).to(dev)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        pieces = [p.cpu().numpy().view(a.dtype)[:per * s].reshape(lead + (s,), order="F")
                  for p, s in zip(parts, sizes)]
        out.append(np.concatenate(pieces, axis=-1) if pieces else a)
    return out


def run_photons_sharded(runner: Callable[..., Accumulator], *, n_photons: int, npos: int = 1,
                        pid_offset: int = 0, group=None, **kw) -> Accumulator:
    """``run_photons_ka`` over the ranks of ``group``: rank r calls
    ``runner(n_photons=count, pid_offset=pid_offset + start, **kw)`` on its
    range and all ranks return the reduced Accumulator, identical to one
    call over all photons."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    start, count = photon_range(n_photons, rank, world, align=npos)
    acc = runner(n_photons=count, pid_offset=pid_offset + start, **kw)
    return reduce_accumulator(acc, group)


def _collective_device(group=None):
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def run_segments_sharded(runner: Callable, *, sources, photons_per_source, segment_of_source,
                         n_segments: int, t0s=None, pid_offset: int = 0, group=None, **kw):
    """``run_segments`` over the ranks of ``group``: rank r transports the
    sources of its contiguous range of whole segments (pid_offset = photons
    before them, segment ids rebased) through
    ``runner(sources=..., photons_per_source=..., segment_of_source=...,
    n_segments=..., t0s=..., pid_offset=..., **kw)`` -> an object or dict
    with maps, tmin, npe and counters; all ranks return (maps, tmin, npe, counters) for all
    segments, identical to one call."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    src = np.asarray(sources, np.float32).reshape(-1, 3)
    cnt, seg = check_segments(photons_per_source, segment_of_source, n_segments)
    if src.shape[0] != cnt.size:
        raise ValueError("sources and photons_per_source differ in length")
    lo, hi, s0, s1, before = shard_segments(cnt, seg, n_segments, rank, world)
    n_local = hi - lo
    pid0 = pid_offset + before
    res = None
    cells_shape = kw.pop("cells_shape", (8, 8))
    if n_local > 0 and s1 > s0:
        res = runner(sources=src[s0:s1], photons_per_source=cnt[s0:s1],
                     segment_of_source=(seg[s0:s1] - lo), n_segments=n_local,
                     t0s=None if t0s is None else np.asarray(t0s, np.float32)[s0:s1],
                     pid_offset=pid0, **kw)
        get = (lambda k: res[k]) if isinstance(res, dict) else (lambda k: getattr(res, k))
        maps, tmin, npe, ctr = get("maps"), get("tmin"), get("npe"), get("counters")
    else:
        maps = np.zeros(tuple(cells_shape) + (n_local,), np.uint32, order="F")
        tmin = np.full(tuple(cells_shape) + (n_local,), np.inf, np.float32, order="F")
        npe = np.zeros(n_local, np.int32)
        ctr = None
    maps_all, tmin_all, npe_all = gather_segments([maps, tmin, npe], n_local, group)
    from .params import COUNTER_NAMES
    dev = _collective_device(group)
    c = torch.tensor([int(ctr[n]) if ctr else 0 for n in COUNTER_NAMES], dtype=torch.int64, device=dev)
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    return maps_all, tmin_all, npe_all, dict(zip(COUNTER_NAMES, (int(v) for v in c.cpu().tolist())))


class ShardedSegments:
    """A segmented job split over the ranks of ``group`` with the inputs of
    this rank's share resident on its GPU: ``step()`` enqueues the transport
    of the share (one ``cl_run_segments_device`` launch sequence, as
    ``batching.DeviceEvents``) and then gathers every rank's per-segment maps,
    first-hit times and npe into device tensors on every rank (NCCL
    all_gather, shares padded to the largest) and sums the counters
    (all_reduce).  The host arrays describing the job are the same on every
    rank; photon ids are numbered over the whole job, so the gathered maps
    equal one single-GPU call bit for bit."""

    def __init__(self, engine, box, op, ro, tb, *, sources, photons_per_source, segment_of_source,
                 n_segments: int, seed: int, tau_ns: float, t0s=None, pid_offset: int = 0,
                 max_bounces: int = 100_000, group=None):
        import torch
        import torch.distributed as dist
        from .batching import DeviceEvents
        self.group = group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        src = np.asarray(sources, np.float32).reshape(-1, 3)
        cnt, seg = check_segments(photons_per_source, segment_of_source, n_segments)
        if src.shape[0] != cnt.size:
            raise ValueError("sources and photons_per_source differ in length")
        self.n_segments = int(n_segments)
        self.plans = [shard_segments(cnt, seg, n_segments, r, self.world) for r in range(self.world)]
        lo, hi, s0, s1, before = self.plans[self.rank]
        self.n_local = hi - lo
        self.n_max = max(p[1] - p[0] for p in self.plans)
        dev = torch.device("cuda", torch.cuda.current_device())
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        t0 = np.zeros(src.shape[0], np.float32) if t0s is None else np.asarray(t0s, np.float32)
        self.local = None
        if self.n_local > 0 and s1 > s0:
            self.local = DeviceEvents(engine, box, op, ro, tb, xyz=T(src[s0:s1]), t0=T(t0[s0:s1]),
                                      photons=T(cnt[s0:s1]), segment=T((seg[s0:s1] - lo).astype(np.int32)),
                                      n_segments=self.n_local, seed=seed, tau_ns=tau_ns,
                                      pid_offset=pid_offset + before, max_bounces=max_bounces)
        self.cells = (ro.grid if hasattr(ro, "grid") else ro).nx * (ro.grid if hasattr(ro, "grid") else ro).ny
        self.n_photons_local = int(cnt[s0:s1].sum())
        # padded send buffers and gathered outputs
        self.send_maps = torch.zeros(self.cells * self.n_max, dtype=torch.int32, device=dev)
        self.send_tmin = torch.full((self.cells * self.n_max,), float("inf"), dtype=torch.float32, device=dev)
        self.send_npe = torch.zeros(self.n_max, dtype=torch.int32, device=dev)
        self.maps_all = torch.empty(self.world * self.cells * self.n_max, dtype=torch.int32, device=dev)
        self.tmin_all = torch.empty(self.world * self.cells * self.n_max, dtype=torch.float32, device=dev)
        self.npe_all = torch.empty(self.world * self.n_max, dtype=torch.int32, device=dev)
        self.counters = torch.zeros(9, dtype=torch.int64, device=dev)

    def step(self, stream=None) -> None:
        """Transport this rank's share, then gather all shares (device work
        only; every rank takes the same collective steps)."""
        import torch
        import torch.distributed as dist
        n = self.cells * self.n_local
        if self.local is not None:
            self.local.step(stream)
            self.send_maps[:n].copy_(self.local.maps)
            self.send_tmin[:n].copy_(self.local.tmin)
            self.send_npe[:self.n_local].copy_(self.local.npe)
            self.counters.copy_(self.local.counters)
        else:
            self.counters.zero_()
        dist.all_gather_into_tensor(self.maps_all, self.send_maps, group=self.group)
        dist.all_gather_into_tensor(self.tmin_all, self.send_tmin, group=self.group)
        dist.all_gather_into_tensor(self.npe_all, self.send_npe, group=self.group)
        dist.all_reduce(self.counters, op=dist.ReduceOp.SUM, group=self.group)

    def sync(self) -> None:
        """Wait for the device and report this rank's transport errors."""
        if self.local is not None:
            self.local.sync()

    def result(self):
        """(maps (nx*ny, n_segments) uint32, tmin, npe, counters dict) on the host,
        the padding of the shares removed."""
        from .params import COUNTER_NAMES
        maps = self.maps_all.cpu().numpy().view(np.uint32).reshape(self.world, self.n_max, self.cells)
        tmin = self.tmin_all.cpu().numpy().reshape(self.world, self.n_max, self.cells)
        npe = self.npe_all.cpu().numpy().reshape(self.world, self.n_max)
        k = [p[1] - p[0] for p in self.plans]
        maps = np.concatenate([maps[r, :k[r]] for r in range(self.world)], axis=0).T
        tmin = np.concatenate([tmin[r, :k[r]] for r in range(self.world)], axis=0).T
        npe = np.concatenate([npe[r, :k[r]] for r in range(self.world)])
        return maps, tmin, npe, dict(zip(COUNTER_NAMES, self.counters.cpu().tolist()))
