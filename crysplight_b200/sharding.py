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
    cnt = np.asarray(photons_per_source, np.int64).reshape(-1)
    seg = np.asarray(segment_of_source, np.int64).reshape(-1)
    per_seg = np.bincount(seg, weights=cnt, minlength=int(n_segments)).astype(np.int64)
    lo, hi, before = segment_range(per_seg, rank, world)
    sel = (seg >= lo) & (seg < hi)
    n_local = hi - lo
    first_src = int(np.argmax(sel)) if sel.any() else 0
    pid0 = pid_offset + int(cnt[:first_src].sum()) if sel.any() else pid_offset + before
    res = None
    cells_shape = kw.pop("cells_shape", (8, 8))
    if n_local > 0 and sel.any():
        res = runner(sources=src[sel], photons_per_source=cnt[sel], segment_of_source=(seg[sel] - lo),
                     n_segments=n_local, t0s=None if t0s is None else np.asarray(t0s, np.float32)[sel],
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
