"""Batched event transport with the deposits resident on the GPU: one launch
sequence (init, transport over prefix-summed photon offsets, finalize) per
batch of events, capturable as a CUDA graph, and an autotuner for the launch
shape.

The reference batches at most ``batch_photons`` photons per kernel launch and
reduces per-photon records on the host (src/events.jl:65-91,
scripts/shoot_gammas.jl:49-54).  Here every photon of every event goes through
one persistent launch whose warps pull photon chunks from a device work queue,
and the per-event maps are reduced on the device.  The launch shape (threads
per CTA, resident CTAs per SM, photons a warp claims from the queue at a time)
does not change any result — each photon's stream is keyed by its global id
and the reductions are exact integer sums and minima — so ``autotune`` may
pick whichever is fastest on a sample of the workload.
"""
from __future__ import annotations

import statistics
from dataclasses import dataclass
from typing import Callable, Iterable

import numpy as np

from .params import Box, OpticalParams, Readout, TimeBinning


@dataclass(frozen=True)
class LaunchShape:
    """Arguments of ``Engine.set_launch`` (0 = automatic)."""
    ctas_per_sm: int = 0
    threads_per_cta: int = 0
    warp_chunk: int = 0


DEFAULT_CANDIDATES = tuple(
    LaunchShape(c, t, w) for t in (256, 128) for c in (0, 3) for w in (32, 64, 128, 256))


def autotune(engine, run_once: Callable[[object], None], *, stream=None,
             candidates: Iterable[LaunchShape] = DEFAULT_CANDIDATES, repeats: int = 3):
    """Time ``run_once(stream)`` under every candidate launch shape (CUDA
    events on ``stream``, median of ``repeats`` after one warm-up run), leave
    the fastest set on ``engine`` and return (best, {shape: seconds})."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    times = {}
    for shape in candidates:
        engine.set_launch(shape.ctas_per_sm, shape.threads_per_cta, shape.warp_chunk)
        run_once(st)
        engine.sync(st.cuda_stream)
        t = []
        for _ in range(repeats):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            run_once(st)
            b.record(st)
            b.synchronize()
            t.append(a.elapsed_time(b) * 1e-3)
        engine.sync(st.cuda_stream)
        times[shape] = statistics.median(t)
    best = min(times, key=times.get)
    engine.set_launch(best.ctas_per_sm, best.threads_per_cta, best.warp_chunk)
    return best, times


class DeviceEvents:
    """A batch of events whose deposits live in HBM, with its output buffers.

    ``step(stream)`` enqueues the whole transport of the batch (no host
    synchronisation, no allocation); ``capture()`` records one step in a CUDA
    graph and ``replay()`` re-launches it; ``result()`` copies the maps back.
    Inputs are CUDA tensors: xyz (n, 3) float32 mm, t0 (n,) float32 ns,
    photons (n,) int64, segment (n,) int32 non-decreasing in [0, n_segments)."""

    def __init__(self, engine, box: Box, op: OpticalParams, ro, tb: TimeBinning, *, xyz, t0, photons,
                 segment, n_segments: int, seed: int, tau_ns: float, pid_offset: int = 0,
                 max_bounces: int = 100_000):
        import torch
        self.engine, self.box, self.op, self.tb = engine, box, op, tb
        self.ro = ro if isinstance(ro, Readout) else Readout(ro)
        dev = xyz.device
        self.sx, self.sy, self.sz = (xyz[:, i].contiguous() for i in range(3))
        self.t0 = t0.contiguous()
        self.seg = segment.contiguous().to(torch.int32)
        self.off = torch.zeros(photons.shape[0] + 1, dtype=torch.int64, device=dev)
        torch.cumsum(photons.to(torch.int64), 0, out=self.off[1:])
        self.n_src = int(photons.shape[0])
        self.n_photons = int(self.off[-1].item())
        self.n_segments = int(n_segments)
        self.seed, self.tau_ns, self.pid_offset, self.max_bounces = seed, tau_ns, pid_offset, max_bounces
        cells = self.ro.grid.nx * self.ro.grid.ny
        self.maps = torch.empty(cells * self.n_segments, dtype=torch.int32, device=dev)
        self.tmin = torch.empty(cells * self.n_segments, dtype=torch.float32, device=dev)
        self.npe = torch.empty(self.n_segments, dtype=torch.int32, device=dev)
        self.counters = torch.empty(9, dtype=torch.int64, device=dev)
        self.graph = None
        self._graph_stream = None

    def step(self, stream=None) -> None:
        import torch
        st = stream if stream is not None else torch.cuda.current_stream()
        self.engine.run_segments_device(
            self.box, self.op, self.ro, self.tb, sx=self.sx.data_ptr(), sy=self.sy.data_ptr(),
            sz=self.sz.data_ptr(), st=self.t0.data_ptr(), src_offsets=self.off.data_ptr(),
            src_segment=self.seg.data_ptr(), n_src=self.n_src, n_segments=self.n_segments,
            n_photons=self.n_photons, seed=self.seed, pid_offset=self.pid_offset, tau_ns=self.tau_ns,
            max_bounces=self.max_bounces, maps=self.maps.data_ptr(), tmin=self.tmin.data_ptr(),
            npe=self.npe.data_ptr(), counters=self.counters.data_ptr(), stream=st.cuda_stream)

    def capture(self) -> None:
        """Record one step in a CUDA graph (warm up first, outside capture)."""
        import torch
        s = torch.cuda.Stream(device=self.maps.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.step(s)
        self.engine.sync(s.cuda_stream)
        g = torch.cuda.CUDAGraph()
        # relaxed: the launch path queries occupancy (no stream work) while capturing
        with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
            self.step(s)
        self.graph, self._graph_stream = g, s

    def replay(self) -> None:
        """Launch the captured step on the current stream."""
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()

    def sync(self, stream=None) -> None:
        """Wait for the device and report the transport's error word."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream()
        torch.cuda.synchronize(self.maps.device)
        self.engine.sync(st.cuda_stream)

    def result(self):
        """(maps (nx, ny, n) uint32 Fortran, tmin, npe, counters dict)."""
        from .params import COUNTER_NAMES
        nx, ny = self.ro.grid.nx, self.ro.grid.ny
        n = self.n_segments
        maps = self.maps.cpu().numpy().view(np.uint32).reshape((nx, ny, n), order="F")
        tmin = self.tmin.cpu().numpy().reshape((nx, ny, n), order="F")
        return maps, tmin, self.npe.cpu().numpy(), dict(zip(COUNTER_NAMES, self.counters.cpu().tolist()))
