"""Pins the CPU oracle against every known answer of the reference's own test
suite (test/runtests.jl) plus the published Philox4x32-10 known-answer
vectors and the reference's published physics results.  No GPU needed."""
import math

import numpy as np
import pytest

from crysplight_b200.params import (Accumulator, Box, OpticalParams, Readout, SipmGrid,
                                    TimeBinning, FACE_BACK, FACE_FRONT, FACE_XM, FACE_XP,
                                    FACE_YM, FACE_YP, STATUS_ABS_SUR, STATUS_DETECTED,
                                    deg2rad_f32, surface_has_gap)
from cases import (BOX_BGO, BOX_CSI, CENTRE_CSI, GRID, INF, OP_ALL, OP_CSI_TEFLON, RO_ALL, TB, TB80,
                   TAU_CSI, ideal)


def test_configuration_validation():            # test/runtests.jl:11-15
    assert surface_has_gap("backpainted")
    assert not surface_has_gap("frontpainted")
    with pytest.raises(ValueError):
        surface_has_gap("back-painted")


# ---- Philox ------------------------------------------------------------------------
KAT = [  # Philox4x32-10 known-answer vectors (Salmon et al., SC'11, Random123 distribution)
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_philox_known_answers(oracle, ctr, key, expect):
    assert oracle.philox4x32(ctr, key) == expect


def test_philox_stream_contract(oracle):          # test/runtests.jl:23-33
    s1, s2 = oracle.PhiloxStream(42, 7), oracle.PhiloxStream(42, 7)
    assert [s1.randu() for _ in range(100)] == [s2.randu() for _ in range(100)]
    assert oracle.PhiloxStream(42, 8).randu() != oracle.PhiloxStream(43, 7).randu()
    u = oracle.randu_streams(1, 200_000, 1)[:, 0].astype(np.float64)
    assert np.all((u > 0) & (u <= 1))
    assert abs(u.mean() - 0.5) < 3e-3
    assert abs(u.std(ddof=1) - math.sqrt(1 / 12)) < 3e-3


def test_philox_stream_keying(oracle):
    """key = (seed lo, seed hi), counter = (pid lo, pid hi, block, 0); first
    block is 0; randu = ((x >> 8) + 1) 2^-24 (src/philox.jl:43-62)."""
    seed, pid = 0x0123456789ABCDEF, 0xFEDCBA9876543210
    s = oracle.PhiloxStream(seed, pid)
    key = (seed & 0xFFFFFFFF, seed >> 32)
    b0 = oracle.philox4x32((pid & 0xFFFFFFFF, pid >> 32, 0, 0), key)
    b1 = oracle.philox4x32((pid & 0xFFFFFFFF, pid >> 32, 1, 0), key)
    assert [s.next_u32() for _ in range(8)] == list(b0 + b1)
    s = oracle.PhiloxStream(5, 9)
    x = oracle.philox4x32((9, 0, 0, 0), (5, 0))[0]
    assert s.randu() == np.float32(((x >> 8) + 1) * 2.0 ** -24)


# ---- geometry ---------------------------------------------------------------------
def test_wall_hit(oracle):                         # test/runtests.jl:35-46
    box = BOX_CSI
    d, f = oracle.wall_hit(24, 24, 18.6, 1, 0, 0, box)
    assert d == pytest.approx(24) and f == FACE_XP
    d, f = oracle.wall_hit(24, 24, 18.6, 0, -1, 0, box)
    assert d == pytest.approx(24) and f == FACE_YM
    d, f = oracle.wall_hit(24, 24, np.float32(18.6), 0, 0, 1, box)
    assert d == pytest.approx(np.float32(37.2) - np.float32(18.6)) and f == FACE_BACK
    u = float(np.float32(1) / np.sqrt(np.float32(2)))
    d, f = oracle.wall_hit(0, 0, 0, u, 0, u, box)
    assert f == FACE_BACK and d == pytest.approx(37.2 * math.sqrt(2), rel=1e-6)


def test_wall_hit_tie_break(oracle):
    # dx <= dy && dx <= dz -> x face first; then dy <= dz -> y (src/geometry.jl:27-31)
    box = Box((10, 10, 10))
    c = float(np.float32(1 / math.sqrt(3)))
    assert oracle.wall_hit(5, 5, 5, c, c, c, box)[1] == FACE_XP
    assert oracle.wall_hit(5, 5, 5, 0, -c, -c, box)[1] == FACE_YM
    assert oracle.wall_hit(5, 5, 5, 0, 0, -1, box)[1] == FACE_FRONT
    assert oracle.wall_hit(5, 5, 5, -1, 0, 0, box)[1] == FACE_XM
    assert oracle.wall_hit(5, 5, 5, 0, 1, 0, box)[1] == FACE_YP


# ---- Fresnel ------------------------------------------------------------------------
def test_fresnel(oracle):                          # test/runtests.jl:48-63
    r0 = ((1.95 - 1.45) / (1.95 + 1.45)) ** 2
    tir, R = oracle.fresnel(1.95, 1.45, 1.0)
    assert not tir and R == pytest.approx(r0, rel=1e-5)
    c40 = float(np.cos(np.float32(40) * (np.float32(math.pi) / np.float32(180))))
    c20 = float(np.cos(np.float32(20) * (np.float32(math.pi) / np.float32(180))))
    assert oracle.fresnel(1.95, 1.0, c40)[0]
    assert not oracle.fresnel(1.95, 1.0, c20)[0]
    assert oracle.fresnel(1.95, 1.45, 1e-4)[1] > 0.999
    tir, Ra = oracle.fresnel(1.45, 1.95, 1.0)
    assert Ra == pytest.approx(r0, rel=1e-5)


# ---- sampling distributions ------------------------------------------------------
def test_sampling_distributions(oracle):           # test/runtests.jl:65-100
    s = oracle.PhiloxStream(7, 1)
    dirs = np.array([oracle.isotropic_dir(s) for _ in range(200_000)], dtype=np.float64)
    assert abs(dirs[:, 2].mean()) < 5e-3
    assert abs((dirs[:, 2] ** 2).mean() - 1 / 3) < 3e-3
    assert np.all(np.abs((dirs[:1000] ** 2).sum(1) - 1) < 1e-5)
    lam = np.array([oracle.lambertian_dir(s, FACE_BACK) for _ in range(200_000)])
    assert np.all(lam[:, 2] < 0)
    assert abs((-lam[:, 2]).mean() - 2 / 3) < 3e-3
    lam = np.array([oracle.lambertian_dir(s, FACE_XM) for _ in range(1000)])
    assert np.all(lam[:, 0] > 0)
    dt = np.array([oracle.emission_time(s, 800.0) for _ in range(200_000)])
    assert dt.mean() == pytest.approx(800, rel=0.01)
    assert oracle.emission_time(s, 0.0) == 0.0
    mus = np.array([oracle.rayleigh_dir(s, 0.0, 0.0, 1.0)[2] for _ in range(200_000)])
    assert abs(mus.mean()) < 6e-3
    assert abs((mus ** 2).mean() - 0.4) < 5e-3
    for _ in range(1000):
        v = np.array(oracle.rayleigh_dir(s, 0.6, 0.64, 0.48), dtype=np.float64)
        assert abs((v ** 2).sum() - 1) < 1e-5
    u = (0.5, 0.5, float(np.sqrt(np.float32(0.5))))
    rx, ry, rz, tr = oracle.surface_interact(s, *u, FACE_XP, 1.95, 1e-6)
    assert not tr and abs(rx + u[0]) < 1e-3 and abs(ry - u[1]) < 1e-3
    res = [oracle.surface_interact(s, *u, FACE_XP, 1.95, deg2rad_f32(12)) for _ in range(2000)]
    assert all(r[3] or r[0] < 0 for r in res)
    assert any(r[3] for r in res)


def test_lambertian_faces_point_inward(oracle):
    s = oracle.PhiloxStream(3, 3)
    axis = {FACE_XP: (0, -1), FACE_XM: (0, 1), FACE_YP: (1, -1), FACE_YM: (1, 1),
            FACE_BACK: (2, -1), FACE_FRONT: (2, 1)}
    for face, (a, sgn) in axis.items():
        for _ in range(200):
            assert oracle.lambertian_dir(s, face)[a] * sgn > 0


# ---- transport anchors ------------------------------------------------------------
def test_transport_conservation_and_limits(oracle):   # test/runtests.jl:102-174
    op = ideal(1.95, wrap_R=0.99, abs_len=500.0, pde=0.4)
    acc = oracle.run_photons(BOX_CSI, op, GRID, TB, n_photons=100_000, seed=1, pos=CENTRE_CSI,
                             tau_ns=800.0)
    assert acc.ndet + acc.nabs_bulk + acc.nabs_wall + acc.nabs_sipm + acc.ncap == 100_000
    assert acc.counts.sum() == acc.ndet

    nl = 50_000
    acc = oracle.run_photons(BOX_CSI, ideal(1.95), GRID, TB, n_photons=nl, seed=2,
                             pos=CENTRE_CSI, tau_ns=0.0, max_bounces=20_000)
    assert acc.ndet + acc.ncap == nl
    assert acc.nabs_bulk == acc.nabs_wall == acc.nabs_sipm == 0
    pc = 1 - math.cos(math.asin(1.45 / 1.95))
    assert acc.ndet / nl > pc - 4 * math.sqrt(pc * (1 - pc) / nl)
    assert acc.ndet < nl

    n = 200_000
    acc = oracle.run_photons(BOX_BGO, ideal(2.15, spec=True), GRID, TB, n_photons=n, seed=3,
                             pos=(24.0, 24.0, 11.2), tau_ns=0.0, max_bounces=20_000)
    p = 1 - math.cos(math.asin(1.45 / 2.15))         # exact escape cone
    assert abs(acc.ndet / n - p) <= 4 * math.sqrt(p * (1 - p) / n)
    assert acc.ncap + acc.ndet == n

    op = ideal(1.95, wrap_R=0.0, abs_len=100.0)
    acc = oracle.run_photons(BOX_CSI, op, GRID, TB, n_photons=50_000, seed=4, pos=CENTRE_CSI,
                             tau_ns=0.0)
    assert acc.total_terminated() == 50_000
    assert acc.nabs_bulk > 0 and acc.nabs_wall > 0

    acc = oracle.run_photons(BOX_CSI, ideal(1.95, ray=100.0), GRID, TB, n_photons=20_000, seed=5,
                             pos=CENTRE_CSI, tau_ns=0.0)
    assert acc.ndet == 20_000 and acc.nscat > 0

    n0 = oracle.run_photons(BOX_CSI, ideal(1.95), GRID, TB, n_photons=30_000, seed=6,
                            pos=CENTRE_CSI, tau_ns=0.0, max_bounces=20_000).ndet
    n1 = oracle.run_photons(BOX_CSI, ideal(1.95, sigma=deg2rad_f32(6)), GRID, TB,
                            n_photons=30_000, seed=6, pos=CENTRE_CSI, tau_ns=0.0,
                            max_bounces=20_000).ndet
    assert n1 > n0

    acc = oracle.run_photons(BOX_CSI, ideal(1.95, gap=False), GRID, TB, n_photons=20_000, seed=7,
                             pos=CENTRE_CSI, tau_ns=0.0)
    assert acc.ndet == 20_000

    acc = oracle.run_photons(BOX_CSI, OP_ALL, GRID, TB, n_photons=100_000, seed=8,
                             pos=CENTRE_CSI, tau_ns=800.0)
    assert acc.total_terminated() == 100_000
    assert acc.counts.sum() == acc.ndet


def test_readout_modes(oracle):                     # test/runtests.jl:176-222
    op = ideal(1.95)
    ro = Readout(GRID, center=(24, 24), radius=10, sur_R=0)
    acc = oracle.OracleAccumulator(GRID, TB)
    s = oracle.PhiloxStream(21, 1)
    assert oracle.propagate_photon(acc, BOX_CSI, op, ro, TB, s, 24, 24, 0, 0, 0, 1, 0)[0] \
        == STATUS_DETECTED
    assert oracle.propagate_photon(acc, BOX_CSI, op, ro, TB, s, 4, 4, 0, 0, 0, 1, 0)[0] \
        == STATUS_ABS_SUR
    assert acc.acc.nabs_sur == 1

    ro = Readout(GRID, center=(24, 24), radius=10, sur_R=0.95)
    opb = ideal(1.79, wrap_R=0.9, abs_len=300.0)
    acc = oracle.run_photons(BOX_CSI, opb, ro, TB, n_photons=50_000, seed=22,
                             pos=(24.0, 24.0, 18.0), tau_ns=0.0)
    assert acc.total_terminated() == 50_000
    assert acc.nabs_sur > 0 and acc.ndet > 0

    ps = [(24.0, 24.0, 5.0), (24.0, 24.0, 30.0)]
    a1 = oracle.run_photons(BOX_CSI, opb, ro, TB, n_photons=20_000, seed=23, positions=ps,
                            tau_ns=0.0)
    a2 = oracle.run_photons(BOX_CSI, opb, ro, TB, n_photons=20_000, seed=23, positions=ps,
                            tau_ns=0.0, nthreads=3)
    assert a1.total_terminated() == 20_000
    assert a1.ndet == a2.ndet and np.array_equal(a1.counts, a2.counts)

    ro2 = Readout(GRID, two_sided=True)
    acc = oracle.OracleAccumulator(GRID, TB)
    s = oracle.PhiloxStream(31, 1)
    assert oracle.propagate_photon(acc, BOX_CSI, ideal(1.95), ro2, TB, s, 24, 24, 18, 0, 0, 1,
                                   0)[0] == STATUS_DETECTED
    assert oracle.propagate_photon(acc, BOX_CSI, ideal(1.95), ro2, TB, s, 24, 24, 18, 0, 0, -1,
                                   0)[0] == STATUS_DETECTED
    assert acc.acc.ndet == 2 and acc.acc.ndet_front == 1
    acc = oracle.run_photons(BOX_CSI, opb, ro2, TB, n_photons=50_000, seed=32, pos=CENTRE_CSI,
                             tau_ns=0.0)
    assert acc.total_terminated() == 50_000
    assert abs(acc.ndet_front / acc.ndet - 0.5) < 0.02


def test_kernel_twin_bit_parity(oracle):            # test/runtests.jl:224-246
    kw = dict(n_photons=100_000, seed=8, pos=CENTRE_CSI, tau_ns=800.0)
    for ro in (RO_ALL, Readout(GRID, two_sided=True)):
        a = oracle.run_photons(BOX_CSI, OP_ALL, ro, TB, **kw)
        b = oracle.run_photons_ka(BOX_CSI, OP_ALL, ro, TB, **kw)
        assert np.array_equal(a.counts, b.counts)
        assert np.array_equal(a.first_ns, b.first_ns)
        assert a.counters() == b.counters()


def test_detection_record(oracle):                  # test/runtests.jl:341-357
    op = ideal(1.95)
    acc = oracle.OracleAccumulator(GRID, TB)
    s = oracle.PhiloxStream(11, 1)
    st, _ = oracle.propagate_photon(acc, BOX_CSI, op, GRID, TB, s, 9, 39, 0, 0, 0, 1, 0)
    assert st == STATUS_DETECTED
    assert acc.acc.counts[1, 6, 0] == 1
    texp = np.float32(37.2) * np.float32(1.95) / np.float32(299.792458)
    assert acc.acc.first_ns[1, 6] == pytest.approx(texp, rel=1e-4)
    st, _ = oracle.propagate_photon(acc, BOX_CSI, op, GRID, TB, s, 9, 39, 0, 0, 0, 1, 1e6)
    assert acc.acc.counts[1, 6, -1] == 1


def test_published_physics_csitl_teflon(oracle):
    """latex/csitl_calib.tex:300-308: CsI(Tl)+Teflon centre, PDE 1: 88.8%
    detected, 10.0% bulk, 1.2% wall (quoted to 0.1%)."""
    n = 400_000
    acc = oracle.run_photons(BOX_CSI, OP_CSI_TEFLON, GRID, TB80, n_photons=n, seed=1234,
                             pos=CENTRE_CSI, tau_ns=TAU_CSI)
    assert abs(acc.ndet / n - 0.888) < 0.0015
    assert abs(acc.nabs_bulk / n - 0.100) < 0.0015
    assert abs(acc.nabs_wall / n - 0.012) < 0.0015
    assert acc.total_terminated() == n


def test_published_physics_bgo_esr(oracle):
    """latex/csitl_calib.tex:470: BGO+ESR, 48x48x22.4, centre, PDE 1: 70.0%."""
    n = 200_000
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, deg2rad_f32(1.3), 1.0)
    acc = oracle.run_photons(BOX_BGO, op, GRID, TB80, n_photons=n, seed=1234,
                             pos=(24.0, 24.0, 11.2), tau_ns=1768.0)
    assert abs(acc.ndet / n - 0.700) < 0.01
