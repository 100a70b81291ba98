"""The allocation-free entry point, cl_run_photons_noalloc.

Some callers cannot let a library call cudaMalloc: programs whose device
memory belongs to a pool or caching allocator (CUDA.jl's, PyTorch's) or to a
fixed budget, and latency-sensitive loops where cudaMalloc/cudaFree would
synchronise the device.  cl_run_photons_noalloc serves them from one static
device array of CL_NOALLOC_SCRATCH_BYTES.  This test calls it through the
C-ABI twice in a row and requires results identical (the same exact equality
the other parity tests use for counts, first-hit time bits and counters) to
the regular entry point cl_run_photons, then checks that an oversized request
is refused with a clear message.  The file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from crysplight_b200 import _lib
from crysplight_b200.params import Accumulator, Counters, Readout, TimeBinning
from cases import BOX_CSI, CENTRE_CSI, GRID, OP_ALL, OP_CSI_TEFLON, RO_ALL, TAU_CSI, TB, TB80

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 1 << 20   # CL_NOALLOC_SCRATCH_BYTES


def _noalloc(box, op, ro, tb, *, n_photons, seed, positions, t0s=None, pid_offset=0, tau_ns,
             max_bounces=100_000):
    lib = _lib.load()
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    p = np.ascontiguousarray(np.asarray(positions, np.float32).reshape(-1, 3))
    px, py, pz = (np.ascontiguousarray(p[:, i]) for i in range(3))
    pt = None if t0s is None else np.ascontiguousarray(np.asarray(t0s, np.float32))
    acc = Accumulator.empty(ro.grid, tb)
    ctr = Counters()
    ptr = lambda a: None if a is None else C.c_void_p(a.ctypes.data)
    rc = lib.cl_run_photons_noalloc(
        C.byref(box), C.byref(op), C.byref(ro), C.byref(tb), ptr(px), ptr(py), ptr(pz), ptr(pt),
        p.shape[0], n_photons, seed, pid_offset, float(np.float32(tau_ns)), max_bounces,
        ptr(acc.counts), ptr(acc.first_ns), C.byref(ctr), None)
    msg = lib.cl_last_error(None).decode()
    if rc == _lib.CL_OK:
        acc.set_counters(ctr)
    return rc, msg, acc


def _same(a, b):
    assert np.array_equal(a.counts, b.counts)
    assert np.array_equal(a.first_ns.view(np.uint32), b.first_ns.view(np.uint32))
    assert a.counters() == b.counters()


def test_noalloc_matches_regular_entry_point_twice(engine):
    calls = [
        (BOX_CSI, OP_CSI_TEFLON, Readout(GRID), TB80,
         dict(n_photons=200_000, seed=1234, positions=[CENTRE_CSI], tau_ns=TAU_CSI)),
        (BOX_CSI, OP_ALL, RO_ALL, TB,
         dict(n_photons=100_000, seed=8, positions=[(24.0, 24.0, 5.0), (24.0, 24.0, 30.0)],
              t0s=[0.0, 40.0], pid_offset=777, tau_ns=800.0)),
    ]
    for box, op, ro, tb, kw in calls:          # two calls in a row on the shared array
        rc, msg, got = _noalloc(box, op, ro, tb, **kw)
        assert rc == _lib.CL_OK, msg
        ref = engine.run_photons_ka(box, op, ro, tb, n_photons=kw["n_photons"], seed=kw["seed"],
                                    positions=kw["positions"], t0s=kw.get("t0s"),
                                    pid_offset=kw.get("pid_offset", 0), tau_ns=kw["tau_ns"])
        _same(got, ref)
        assert got.total_terminated() == kw["n_photons"]


def test_noalloc_refuses_requests_larger_than_its_array(engine):
    big = TimeBinning(1.0, SCRATCH_BYTES // (4 * 64))   # 64 cells x (nbins+1) words > 1 MiB
    rc, msg, _ = _noalloc(BOX_CSI, OP_CSI_TEFLON, GRID, big, n_photons=10, seed=1,
                          positions=[CENTRE_CSI], tau_ns=0.0)
    assert rc == _lib.CL_ERR_ARG
    assert "static device array" in msg
    # the array is still usable afterwards, and a later call leaves nothing behind
    rc, msg, a = _noalloc(BOX_CSI, OP_CSI_TEFLON, GRID, TB, n_photons=5_000, seed=3,
                          positions=[CENTRE_CSI], tau_ns=0.0)
    assert rc == _lib.CL_OK, msg
    ref = engine.run_photons_ka(BOX_CSI, OP_CSI_TEFLON, GRID, TB, n_photons=5_000, seed=3,
                                pos=CENTRE_CSI, tau_ns=0.0)
    _same(a, ref)
