"""Surrogate training data: the point scan with arrival-time moments.

The moment sums of cl_run_segments_moments_device are exact integer sums of
per-photon fixed-point values, so they are checked bit for bit against the
same sums formed from per-photon records of the plain segment path (whose
records the oracle parity tests pin), and the counts and first-hit times of
the two paths must be identical."""
import numpy as np
import pytest

from cases import BOX_BGO, BOX_CSI, GRID, OP_CSI_TEFLON, OP_BGO_ESR, TB80, scan_points

pytestmark = pytest.mark.gpu


def _fixed_sums(recs, per, n_points, cells):
    from crysplight_b200 import _lib
    from crysplight_b200.params import STATUS_DETECTED
    det = recs.status == STATUS_DETECTED
    k = np.nonzero(det)[0]
    cell = np.abs(recs.idx[k].astype(np.int64)) - 1
    slot = (k // per) * cells + cell
    tc = np.clip(recs.t[k].astype(np.float32), np.float32(0), np.float32(_lib.MOMENT_T_MAX_NS))
    f1 = np.rint(tc * np.float32(_lib.MOMENT_T_SCALE)).astype(np.uint64)
    f2 = np.rint((tc * tc).astype(np.float32) * np.float32(_lib.MOMENT_T2_SCALE)).astype(np.uint64)
    s1 = np.zeros(n_points * cells, np.uint64)
    s2 = np.zeros(n_points * cells, np.uint64)
    np.add.at(s1, slot, f1)
    np.add.at(s2, slot, f2)
    cnt = np.bincount(slot, minlength=n_points * cells)
    return cnt.reshape(n_points, cells), s1.reshape(n_points, cells), s2.reshape(n_points, cells)


@pytest.mark.parametrize("case", ["bgo_esr", "csitl_teflon"])
def test_scan_moments_exact(engine, case):
    from crysplight_b200.surrogate import scan_light
    box, op = (BOX_BGO, OP_BGO_ESR) if case == "bgo_esr" else (BOX_CSI, OP_CSI_TEFLON)
    pts = scan_points(6, box, seed=5)
    per = 4000
    scan = scan_light(engine, box, op, GRID, points=pts, photons_per_point=per, seed=21,
                      pid_offset=77, batch_points=4)
    res, rec = engine.run_segments(box, op, GRID, TB80, sources=pts, photons_per_source=[per] * 6,
                                   segment_of_source=range(6), n_segments=6, seed=21, pid_offset=77,
                                   tau_ns=0.0, return_records=True)
    cells = 64
    maps = res.maps.reshape(cells, 6, order="F").T
    tmin = res.tmin.reshape(cells, 6, order="F").T
    assert np.array_equal(scan.counts, maps.astype(np.int64))
    assert np.array_equal(scan.tmin.view(np.uint32), tmin.view(np.uint32))
    cnt, s1, s2 = _fixed_sums(rec, per, 6, cells)
    assert np.array_equal(cnt, scan.counts)
    assert np.array_equal(s1, scan.tsum)
    assert np.array_equal(s2, scan.tsum2)
    assert scan.counters["ndet"] == int(maps.sum())


def test_targets_from_scan(engine):
    from crysplight_b200.surrogate import light_targets, scan_light
    pts = scan_points(4, BOX_BGO, seed=9)
    scan = scan_light(engine, BOX_BGO, OP_BGO_ESR, GRID, points=pts, photons_per_point=50_000, seed=3)
    y = light_targets(scan)
    assert y.shape == (4, 192) and np.isfinite(y).all()
    p = np.exp(y[:, :64])
    assert np.allclose(p.sum(1), scan.counts.sum(1) / 50_000, rtol=0.05)
    # mean transit time from the moments vs the first-hit time: mean >= first
    ok = scan.counts >= 100
    assert (y[:, 64:128][ok] >= scan.tmin[ok] - 1e-3).all()
