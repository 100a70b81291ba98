"""The surrogate's first-pass term on the GPU: cl_surrogate_direct against its
NumPy restatement (oracle/first_pass.py, itself checked against the reference
transport's unscattered detections in tests/test_first_pass.py), its argument
checks, and cl_surrogate_combine_direct, which adds the term to an ensemble
trained on the light response minus it."""
import ctypes as C

import numpy as np
import pytest

from crysplight_b200 import _lib
from crysplight_b200.params import Box, OpticalParams, Readout, SipmGrid
from oracle import first_pass as FP

pytestmark = pytest.mark.gpu

GRID = SipmGrid(6.0, 8, 8)


def _direct_gpu(xyz, box, op, ro):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(xyz, np.float32)).cuda()
    out = torch.full((x.shape[0], 64), -1.0, dtype=torch.float32, device="cuda")
    rc = _lib.load().cl_surrogate_direct(C.c_void_p(x.data_ptr()), int(x.shape[0]), C.byref(box), C.byref(op),
                                         C.byref(ro), C.c_void_p(out.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("name, box, op", [
    ("bgo_esr", (48.0, 48.0, 22.4), OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, 0.0227, 1.0)),
    ("csitl_teflon", (48.0, 48.0, 37.2), OpticalParams(1.79, 1.45, 3115.0, 346.0, 0.99, False, True, 0.0227, 1.0)),
    ("ideal", (30.0, 42.0, 12.0), OpticalParams(1.82, 1.0, float("inf"), float("inf"), 1.0, True, True, 0.0, 1.0)),
])
def test_direct_matches_restatement(name, box, op):
    rng = np.random.default_rng(3)
    L = np.array(box)
    n = 3000
    xyz = rng.uniform(0, 1, (n, 3)) * L
    xyz[:, 2] = L[2] * (1.0 - rng.uniform(0.0005, 0.6, n))   # near and far from the readout face
    xyz[:8] = [[L[0] / 2, L[1] / 2, L[2] - 0.5], [6.0, 6.0, L[2] - 1.0], [0.3, 0.3, L[2] - 0.3],
               [L[0] / 2, L[1] / 2, L[2]], [L[0] / 2, L[1] / 2, L[2] + 1.0], [-1.0, 3.0, 1.0],
               [L[0], L[1], L[2] - 2.0], [L[0] / 2, 0.0, 0.0]]
    xyz = xyz.astype(np.float32)
    ro = Readout(GRID)
    got = _direct_gpu(xyz, Box(box), op, ro)
    # the box as the kernel sees it (Float32): a site on the face has h = 0 there
    want = FP.direct(xyz.astype(np.float64), [float(v) for v in np.float32(box)], float(op.n_crystal),
                     float(op.n_coupling),
                     float(op.abs_len_mm), float(op.rayleigh_mm), 6.0, 8, 8)
    err = np.abs(got - want)
    assert np.all(err <= 2e-4 * want + 2e-6), (name, float(err.max()), int(err.argmax()))
    assert np.all(got[3:6] == 0.0)      # on / beyond the readout face, outside the crystal


def test_direct_argument_checks():
    import torch
    lib = _lib.load()
    x = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    out = torch.empty((4, 64), dtype=torch.float32, device="cuda")
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, 0.0227, 1.0)
    P = C.c_void_p

    def call(ro, op=op, n=4):
        return lib.cl_surrogate_direct(P(x.data_ptr()), n, C.byref(Box((48.0, 48.0, 22.4))), C.byref(op),
                                       C.byref(ro), P(out.data_ptr()), None)
    assert call(Readout(GRID)) == _lib.CL_OK
    assert call(Readout(SipmGrid(6.0, 4, 4))) == _lib.CL_ERR_ARG          # 16 cells
    assert call(Readout(GRID, two_sided=True)) == _lib.CL_ERR_ARG         # a second readout face
    assert call(Readout(GRID, center=(24.0, 24.0), radius=10.0)) == _lib.CL_ERR_ARG   # a disc readout
    assert call(Readout(GRID), op=OpticalParams(2.15, 1.45, -1.0, 2222.0, 0.985, True, True, 0.0, 1.0)) == \
        _lib.CL_ERR_ARG
    assert call(Readout(GRID), n=0) == _lib.CL_OK


def test_combine_direct_adds_the_term_to_mean_and_total():
    import torch
    rng = np.random.default_rng(5)
    K, n = 5, 800
    raw = rng.standard_normal((K, n, 192)).astype(np.float32) * 0.05
    y_mean = np.concatenate([np.full(64, -5.5), np.full(64, 3.0), np.full(64, -0.5)]).astype(np.float32)
    y_std = np.concatenate([np.full(64, 0.8), np.full(64, 1.0), np.full(64, 0.2)]).astype(np.float32)
    raw[:, :12, :64] += rng.standard_normal((K, 12, 64)).astype(np.float32) * 0.3
    xyz = (rng.uniform(0.05, 0.95, (n, 3)) * [48, 48, 22.4]).astype(np.float32)
    D = (rng.uniform(0, 1, (n, 64)) ** 8 * 0.05).astype(np.float32)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
         dict(raw=raw, ym=y_mean, ys=y_std, xyz=xyz, D=D).items()}
    out = {k: torch.empty(s, dtype=d, device="cuda") for k, s, d in
           (("p", (n, 64), torch.float32), ("tm", (n, 64), torch.float32), ("ts", (n, 64), torch.float32),
            ("sp", (n,), torch.float32), ("fl", (n,), torch.uint8))}
    P = C.c_void_p
    rc = _lib.load().cl_surrogate_combine_direct(
        P(t["raw"].data_ptr()), K, n, P(t["ym"].data_ptr()), P(t["ys"].data_ptr()), P(t["xyz"].data_ptr()),
        P(t["D"].data_ptr()), C.byref(Box((48.0, 48.0, 22.4))), C.byref(Readout(GRID)), 0.4, 0.02, 1.0,
        P(out["p"].data_ptr()), P(out["tm"].data_ptr()), P(out["ts"].data_ptr()), P(out["sp"].data_ptr()),
        P(out["fl"].data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    o = {k: v.cpu().numpy() for k, v in out.items()}
    y = raw.astype(np.float64) * y_std + y_mean
    p = np.exp(y[:, :, :64])
    total = D.astype(np.float64) + p.mean(0)
    spread = p.std(0).sum(1) / total.sum(1)
    assert np.allclose(o["p"], 0.4 * total, rtol=1e-5)
    assert np.allclose(o["sp"], spread, rtol=1e-4)
    assert np.array_equal(o["fl"] & 1, (spread > 0.02).astype(np.uint8))
    assert (o["fl"][:12] & 1).all()      # the disagreeing members


def test_direct_has_the_same_bits_in_any_batch():
    """A site's first-pass term does not depend on the other sites of the
    call (its contributions are summed as fixed-point integers), so an expert
    evaluated on a subset of the sites gives the main ensemble's bits."""
    rng = np.random.default_rng(9)
    L = (48.0, 48.0, 22.4)
    xyz = (rng.uniform(0, 1, (4000, 3)) * [48.0, 48.0, 8.0] + [0.0, 0.0, 14.4]).astype(np.float32)
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, 0.0227, 1.0)
    full = _direct_gpu(xyz, Box(L), op, Readout(GRID))
    idx = np.sort(rng.choice(4000, 1234, replace=False))
    sub = _direct_gpu(xyz[idx], Box(L), op, Readout(GRID))
    again = _direct_gpu(xyz, Box(L), op, Readout(GRID))
    assert np.array_equal(full[idx], sub) and np.array_equal(full, again)
