"""The device-resident sharded job (sharding.ShardedSegments: each rank's
share transported from its HBM, then NCCL all_gather of maps, first-hit times
and npe and all_reduce of the counters) on one GPU: a one-rank NCCL group runs
the same code path as N ranks, and its gathered outputs equal one
cl_run_segments call bit for bit."""
import os
import socket

import numpy as np
import pytest

from cases import BOX_CSI, GRID, OP_CSI_TEFLON, TB80, scan_points

pytestmark = pytest.mark.gpu


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_segments_on_one_rank_equal_a_single_call(engine):
    import datetime
    import torch
    import torch.distributed as dist
    from crysplight_b200.sharding import ShardedSegments, run_segments_sharded
    pts = scan_points(12, BOX_CSI, seed=4)
    cnt = np.array([3000, 0, 4500, 1200, 8000, 600, 0, 5000, 2500, 900, 7000, 300], np.int64)
    seg = np.array([0, 0, 1, 2, 2, 3, 4, 5, 5, 6, 7, 7], np.int64)
    t0 = np.linspace(0.0, 3.0, 12).astype(np.float32)
    kw = dict(seed=5, tau_ns=1000.0)
    ref = engine.run_segments(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, sources=pts, photons_per_source=cnt,
                              segment_of_source=seg, n_segments=8, t0s=t0, **kw)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(_port())
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
    try:
        job = ShardedSegments(engine, BOX_CSI, OP_CSI_TEFLON, GRID, TB80, sources=pts, photons_per_source=cnt,
                              segment_of_source=seg, n_segments=8, t0s=t0, **kw)
        for _ in range(2):                  # a second step reuses every buffer
            job.step()
        job.sync()
        maps, tmin, npe, ctr = job.result()
        assert np.array_equal(maps, ref.maps.reshape(64, 8, order="F"))
        assert np.array_equal(tmin.view(np.uint32), ref.tmin.reshape(64, 8, order="F").view(np.uint32))
        assert np.array_equal(npe, ref.npe) and ctr == ref.counters
        # the host-buffer form of the same split
        runner = lambda **k: engine.run_segments(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, **kw, **k)
        m2, t2, n2, c2 = run_segments_sharded(runner, sources=pts, photons_per_source=cnt,
                                              segment_of_source=seg, n_segments=8, t0s=t0)
        assert np.array_equal(m2, ref.maps) and np.array_equal(n2, ref.npe) and c2 == ref.counters
        job = None
    finally:
        dist.destroy_process_group()
