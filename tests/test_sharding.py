"""Multi-GPU sharding logic, run on the CPU: two gloo ranks split a point
source and an event batch, each transporting its share with the oracle, and
the reduced / gathered results must equal one single-process run bit for bit
(photon streams are keyed by global photon id, so any partition reproduces
the same photons).  No GPU."""
import os
import socket

import numpy as np
import pytest

from cases import BOX_CSI, GRID, OP_ALL, OP_CSI_TEFLON, TB, TB80, scan_points


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


POINT = dict(n_photons=6001, seed=77, positions=[(24.0, 24.0, 18.6), (10.0, 30.0, 5.0), (40.0, 8.0, 30.0)],
             tau_ns=800.0)


def _events():
    pts = scan_points(12, BOX_CSI, seed=4)
    cnt = np.array([300, 0, 450, 120, 800, 60, 0, 500, 250, 90, 700, 30], np.int64)
    seg = np.array([0, 0, 1, 2, 2, 3, 4, 5, 5, 6, 7, 7], np.int64)
    t0 = np.linspace(0.0, 3.0, 12).astype(np.float32)
    return pts, cnt, seg, 8, t0


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from oracle import oracle
    from crysplight_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        acc = sharding.run_photons_sharded(
            lambda **kw: oracle.run_photons_ka(BOX_CSI, OP_ALL, GRID, TB, nthreads=2, **kw),
            npos=len(POINT["positions"]), **POINT)
        pts, cnt, seg, n_seg, t0 = _events()
        maps, tmin, npe, ctr = sharding.run_segments_sharded(
            lambda **kw: oracle.run_segments(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, nthreads=2, seed=5, tau_ns=1000.0,
                                             **kw),
            sources=pts, photons_per_source=cnt, segment_of_source=seg, n_segments=n_seg, t0s=t0)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), counts=acc.counts, first=acc.first_ns,
                 ctr=np.array([acc.ndet, acc.nabs_bulk, acc.nabs_wall, acc.nscat, acc.sum_bounces_det]),
                 maps=maps, tmin=tmin, npe=npe, ectr=np.array(list(ctr.values())))
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def sharded(tmp_path_factory, oracle):
    import torch.multiprocessing as mp
    out = str(tmp_path_factory.mktemp("shards"))
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    return [dict(np.load(os.path.join(out, f"rank{r}.npz"))) for r in range(2)]


def test_ranges_partition():
    from crysplight_b200.sharding import photon_range, segment_range
    for n, world, align in ((10, 3, 3), (6001, 2, 3), (5, 8, 1), (0, 2, 1)):
        r = [photon_range(n, k, world, align) for k in range(world)]
        assert sum(c for _, c in r) == n
        assert all(r[k][0] + r[k][1] == r[k + 1][0] or r[k + 1][1] == 0 for k in range(world - 1))
        assert all(s % align == 0 for s, c in r if c)
    w = [5, 0, 3, 9, 1, 1]
    r = [segment_range(w, k, 2) for k in range(2)]
    assert r[0][0] == 0 and r[0][1] == r[1][0] and r[1][1] == len(w) and r[1][2] == sum(w[:r[1][0]])


def test_sharded_point_source_equals_single_run(sharded, oracle):
    acc = oracle.run_photons_ka(BOX_CSI, OP_ALL, GRID, TB, nthreads=4, **POINT)
    for r in sharded:
        assert np.array_equal(r["counts"], acc.counts)
        assert np.array_equal(r["first"].view(np.uint32), acc.first_ns.view(np.uint32))
        assert r["ctr"].tolist() == [acc.ndet, acc.nabs_bulk, acc.nabs_wall, acc.nscat, acc.sum_bounces_det]


def test_sharded_events_equal_single_run(sharded, oracle):
    pts, cnt, seg, n_seg, t0 = _events()
    ref = oracle.run_segments(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, sources=pts, photons_per_source=cnt,
                              segment_of_source=seg, n_segments=n_seg, t0s=t0, seed=5, tau_ns=1000.0,
                              nthreads=4)
    for r in sharded:
        assert np.array_equal(r["maps"], ref["maps"])
        assert np.array_equal(r["tmin"].view(np.uint32), ref["tmin"].view(np.uint32))
        assert np.array_equal(r["npe"], ref["npe"])
        assert r["ectr"].tolist() == list(ref["counters"].values())
        assert ref["npe"].sum() > 0 and (ref["npe"] == 0).any()     # segments with and without light


def _reject_worker(rank, world, port, outdir):
    import torch.distributed as dist
    from crysplight_b200 import sharding
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    msgs = []
    try:
        calls = []
        runner = lambda **kw: calls.append(kw)
        pts = np.zeros((4, 3), np.float32)
        for seg, n_seg in (([0, 2, 1, 3], 4), ([0, 1, 1, 5], 4), ([0, -1, 1, 2], 4)):
            try:
                sharding.run_segments_sharded(runner, sources=pts, photons_per_source=[10, 20, 30, 40],
                                              segment_of_source=seg, n_segments=n_seg)
                msgs.append("accepted")
            except ValueError as e:
                msgs.append(str(e))
        # a valid job still goes through afterwards (same collective steps on every rank)
        dist.barrier()
        msgs.append(f"runner calls {len(calls)}")
    finally:
        dist.destroy_process_group()
    with open(os.path.join(outdir, f"rank{rank}.txt"), "w") as f:
        f.write("\n".join(msgs))


def test_sharded_segments_reject_decreasing_segment_ids(tmp_path):
    """Photon ids are numbered segment-major (src/events.jl:70,88): with a
    segment id that decreases along the sources the photons before a rank's
    range are not the photons of the sources before it, so every rank rejects
    the job before any transport or collective."""
    import torch.multiprocessing as mp
    mp.spawn(_reject_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        lines = open(tmp_path / f"rank{r}.txt").read().splitlines()
        assert "non-decreasing" in lines[0]
        assert "out of range" in lines[1] and "out of range" in lines[2]
        assert lines[3] == "runner calls 0"


def test_shard_plans_cover_the_sources_once():
    from crysplight_b200.sharding import check_segments, shard_segments
    pts, cnt, seg, n_seg, t0 = _events()
    for world in (1, 2, 3, 5, 8):
        plans = [shard_segments(cnt, seg, n_seg, r, world) for r in range(world)]
        assert plans[0][0] == 0 and plans[-1][1] == n_seg
        assert plans[0][2] == 0 and plans[-1][3] == len(cnt)
        for a, b in zip(plans, plans[1:]):
            assert a[1] == b[0] and a[3] == b[2]
        for lo, hi, s0, s1, before in plans:
            assert before == int(cnt[:s0].sum())
            assert all(lo <= s < hi for s in seg[s0:s1])
    with pytest.raises(ValueError):
        check_segments([1, 2], [1, 0], 2)
    with pytest.raises(ValueError):
        check_segments([1, -2], [0, 1], 2)


def _fake_trainer(calls):
    def train(k, x, y):
        calls.append(k)
        # a deterministic function of the member index and of the data
        p = (np.arange(181_952, dtype=np.float32) % 97) * np.float32(k + 1) + np.float32(float(x.sum()))
        return p, [float(k), float(k) + 0.5, float(y.mean())]
    return train


def _surrogate_data():
    from crysplight_b200.params import Box
    from crysplight_b200.surrogate import grid_points
    box = Box((48.0, 48.0, 22.4))
    pts = grid_points(box, (4, 4, 3))
    rng = np.random.default_rng(3)
    return box, pts, rng.normal(size=(pts.shape[0], 192)).astype(np.float32)


def _member_worker(rank, world, port, outdir):
    import torch.distributed as dist
    from crysplight_b200.surrogate import LightSurrogate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        box, pts, y = _surrogate_data()
        calls = []
        sur = LightSurrogate.train(box, pts, y, members=5, group=dist.group.WORLD,
                                   member_trainer=_fake_trainer(calls))
        np.savez(os.path.join(outdir, f"m{rank}.npz"), members=np.stack(sur.members),
                 calls=np.array(calls), hist=np.array(sur.meta["loss_history"]))
    finally:
        dist.destroy_process_group()


def test_surrogate_members_one_per_rank(tmp_path):
    """Ensemble members spread over two gloo ranks (rank r trains members r,
    r + 2, ...) and gathered: every rank holds the same ensemble, in member
    order, as one process training all five."""
    import torch.multiprocessing as mp
    from crysplight_b200.surrogate import LightSurrogate, members_of_rank
    assert members_of_rank(5, 0, 2) == [0, 2, 4] and members_of_rank(5, 1, 2) == [1, 3]
    assert members_of_rank(3, 3, 4) == []
    mp.spawn(_member_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    box, pts, y = _surrogate_data()
    calls = []
    ref = LightSurrogate.train(box, pts, y, members=5, member_trainer=_fake_trainer(calls))
    assert calls == [0, 1, 2, 3, 4]
    for r in range(2):
        got = dict(np.load(tmp_path / f"m{r}.npz"))
        assert got["calls"].tolist() == members_of_rank(5, r, 2)
        assert np.array_equal(got["members"], np.stack(ref.members))
        assert np.allclose(got["hist"], np.array(ref.meta["loss_history"]))
