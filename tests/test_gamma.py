"""The host gamma stage of the event pipeline (csrc/cl_gamma.cpp) against the
reference's own tests of its vendored gamma core (test/runtests.jl:258-303)
and its published 50k-event truth statistics
(analysis/results/true_info/gammas_*_50k_stats.txt).  No GPU needed."""
import math

import numpy as np
import pytest

from crysplight_b200.events import (DEP_BELOWCUT, DEP_COMPTON, DEP_PHOTO, GammaMaterial,
                                    gamma_deposits, gamma_stage, load_xcom, rand_poisson)
from crysplight_b200.params import Box


@pytest.fixture(scope="module")
def csi():
    return GammaMaterial.from_csv("CsI", 4.51, "xcom_CSI.csv")


@pytest.fixture(scope="module")
def bgo():
    return GammaMaterial.from_csv("BGO", 7.13, "xcom_BGO.csv")


L_CSI = Box((48.0, 48.0, 37.2))
L_BGO = Box((48.0, 48.0, 22.4))


def test_xcom_loader():
    x = load_xcom(__import__("crysplight_b200").config.PKG_DATA_DIR + "/xcom_CSI.csv")
    assert x["E_MeV"][0] == pytest.approx(0.01)
    assert np.all(np.diff(x["E_MeV"]) >= 0)          # K-edge rows repeat an energy


def test_cross_sections(csi, bgo):                  # test/runtests.jl:263-273
    assert csi.mfp(0.511) == pytest.approx(2.44, rel=0.02)
    assert bgo.mfp(0.511) < csi.mfp(0.511)
    assert csi.sigma_macro(0.03325)[1] > 2 * csi.sigma_macro(0.03310)[1]   # iodine K edge
    assert csi.sigma_macro(0.511)[2] == 0.0
    assert csi.sigma_macro(10.0)[2] > 0.0


def test_vacuum_escapes():                           # test/runtests.jl:275-280
    vac = GammaMaterial.vacuum()
    assert gamma_deposits(vac, L_CSI, (24.0, 24.0, 0.0), seed=1, stream=1) == []


def test_deposits_sanity(csi):                       # test/runtests.jl:282-299
    nin = 0
    for ev in range(1, 201):
        deps = gamma_deposits(csi, L_CSI, (24.0, 24.0, 0.0), seed=7, stream=ev)
        if not deps:
            continue
        nin += 1
        for d in deps:
            assert 0 <= d[0] <= 48 and 0 <= d[1] <= 48 and 0 <= d[2] <= np.float32(37.2)
            assert 0 <= d[4] < 1.0
        assert sum(d[3] for d in deps) <= 511.001
        assert all(d[5] == DEP_COMPTON for d in deps[:-1])
        assert deps[-1][5] in (DEP_PHOTO, DEP_COMPTON, DEP_BELOWCUT)
    assert nin > 100


def test_poisson_moments():                          # test/runtests.jl:301-303
    ps = np.array([rand_poisson(5, i, 20.0) for i in range(1, 20_001)], dtype=np.float64)
    assert ps.mean() == pytest.approx(20, rel=0.02)
    assert ps.var() == pytest.approx(20, rel=0.05)
    big = np.array([rand_poisson(6, i, 400.0) for i in range(1, 20_001)], dtype=np.float64)
    assert big.mean() == pytest.approx(400, rel=0.005)
    assert big.var() == pytest.approx(400, rel=0.05)
    assert rand_poisson(1, 1, 0.0) == 0


def test_truth_record_consistency(csi):              # test/runtests.jl:315-332 (truth part)
    g = gamma_stage(csi, L_CSI, n_events=400, seed=3, yield_per_mev=54_000)
    for ev in range(400):
        assert g.e1[ev] + g.e2[ev] + g.er[ev] == pytest.approx(511.0, abs=0.01)
        assert (g.int_type[ev] == -1) == (g.edep[ev] == 0)
        if g.int_type[ev] == 0:
            assert g.n_int[ev] == 1 and g.e1[ev] == pytest.approx(511.0, abs=0.01)
        if g.int_type[ev] >= 0:
            assert 0 <= g.xyz1[0, ev] <= 48 and 0 <= g.xyz1[2, ev] <= np.float32(37.2)
            assert g.n_int[ev] >= 1 and g.e1[ev] > 0
    # photons: Poisson(54000 * E / 1000) per deposit, in event order
    assert np.all(np.diff(g.dep_event) >= 0)
    sel = g.dep_photons > 0
    ratio = g.dep_photons[sel].sum() / (54.0 * g.edep.sum())
    assert ratio == pytest.approx(1.0, rel=0.01)


@pytest.mark.parametrize("name,box,density,xcom,interacted,contained", [
    # analysis/results/true_info/gammas_csitl_50k_stats.txt, gammas_bgo_50k_stats.txt
    ("CsI", L_CSI, 4.51, "xcom_CSI.csv", 39106 / 50000, 25573 / 50000),
    ("BGO", L_BGO, 7.13, "xcom_BGO.csv", 43395 / 50000, 37819 / 50000),
])
def test_published_50k_statistics(name, box, density, xcom, interacted, contained):
    mat = GammaMaterial.from_csv(name, density, xcom)
    n = 50_000
    g = gamma_stage(mat, box, n_events=n, seed=11, yield_per_mev=1.0)
    f_int = float((g.edep > 0).mean())
    f_cont = float((g.edep > 510.5).mean())
    tol_i = 4 * math.sqrt(interacted * (1 - interacted) / n) * math.sqrt(2)
    tol_c = 4 * math.sqrt(contained * (1 - contained) / n) * math.sqrt(2)
    print(name, f_int, interacted, f_cont, contained)
    assert abs(f_int - interacted) < tol_i
    assert abs(f_cont - contained) < tol_c
