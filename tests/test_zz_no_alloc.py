"""The allocation-free entry point, cl_run_photons_noalloc.

Some callers cannot let a library call cudaMalloc: programs whose device
memory belongs to a pool or caching allocator (CUDA.jl's, PyTorch's) or to a
fixed budget, and latency-sensitive loops where cudaMalloc/cudaFree would
synchronise the device.  cl_run_photons_noalloc serves them from one static
device array of CL_NOALLOC_SCRATCH_BYTES.  This test calls it through the
C-ABI twice in a row and requires results identical (the same exact equality
the other parity tests use for counts, first-hit time bits and counters) to
the regular entry point cl_run_photons, checks that an oversized request is
refused with a clear message, and, in a fresh process, that repeated calls on
the default stream and on a stream the caller created leave the device's free
memory unchanged.  The file is collected last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from crysplight_b200 import _lib
from crysplight_b200.params import Accumulator, Counters, Readout, TimeBinning
from cases import BOX_CSI, CENTRE_CSI, GRID, OP_ALL, OP_CSI_TEFLON, RO_ALL, TAU_CSI, TB, TB80

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 1 << 20   # CL_NOALLOC_SCRATCH_BYTES


def _noalloc(box, op, ro, tb, *, n_photons, seed, positions, t0s=None, pid_offset=0, tau_ns,
             max_bounces=100_000, stream=None):
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
        ptr(acc.counts), ptr(acc.first_ns), C.byref(ctr), None if stream is None else C.c_void_p(stream))
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


def _measure_device_memory() -> dict:
    """Run in a fresh process: free device memory before and after repeated
    calls, on the legacy default stream and on a stream the caller created."""
    import torch
    torch.cuda.set_device(0)
    user = torch.cuda.Stream()
    cfgs = [(BOX_CSI, OP_CSI_TEFLON, Readout(GRID), TB80,
             dict(n_photons=50_000, seed=21, positions=[CENTRE_CSI], tau_ns=TAU_CSI)),
            (BOX_CSI, OP_ALL, RO_ALL, TB,
             dict(n_photons=20_000, seed=8, positions=[(24.0, 24.0, 5.0)], tau_ns=0.0))]
    rcs = []
    for stream in (None, user.cuda_stream):          # warm-up: every kernel loaded once
        for box, op, ro, tb, kw in cfgs:
            rcs.append(_noalloc(box, op, ro, tb, stream=stream, **kw)[0])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    results = []
    for _ in range(3):
        for stream in (None, user.cuda_stream):
            for box, op, ro, tb, kw in cfgs:
                rc, msg, acc = _noalloc(box, op, ro, tb, stream=stream, **kw)
                rcs.append(rc)
                results.append(int(acc.counts.sum()))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return {"rcs": rcs, "free0": int(free0), "free1": int(free1), "sums": results}


def test_noalloc_allocates_no_device_memory():
    """The property the entry point exists for: after a first call per
    configuration, further calls (on the default stream and on a stream the
    caller created) leave the device's free memory unchanged.  Measured in a
    fresh process so that nothing else allocates meanwhile."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--measure"], capture_output=True,
                       text=True, timeout=600, cwd=os.path.dirname(os.path.abspath(__file__)))
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert all(rc == _lib.CL_OK for rc in out["rcs"]), out["rcs"]
    assert out["free1"] == out["free0"], out
    # the repeated calls give the same results on either stream
    s = out["sums"]
    assert s[0::2] == [s[0]] * len(s[0::2]) and s[1::2] == [s[1]] * len(s[1::2])


if __name__ == "__main__" and sys.argv[1:] == ["--measure"]:
    print(json.dumps(_measure_device_memory()))
