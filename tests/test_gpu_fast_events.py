"""Surrogate event generation: the sampler's variates against their exact
distributions, the ensemble reduction against NumPy, the all-fallback path
against the plain segment transport (bit for bit), and sampling from a
high-statistics light response against the Monte Carlo of the same sites."""
import numpy as np
import pytest

from cases import BOX_BGO, GRID, OP_BGO_ESR, TB80, TAU_BGO, scan_points

pytestmark = pytest.mark.gpu


def _draw(fn, par, n, seed=5):
    import torch
    from crysplight_b200 import _lib
    import ctypes as C
    lib = _lib.load()
    out = torch.empty(n, dtype=torch.int64 if fn == 0 else torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    par = np.asarray(list(par) + [0.0] * (4 - len(par)), np.float64)
    rc = lib.cl_debug_sampler(fn, C.c_void_p(par.ctypes.data), n, seed, C.c_void_p(out.data_ptr()),
                              C.c_void_p(err.data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out.cpu().numpy()


@pytest.mark.parametrize("n,p", [(5, 0.3), (40, 0.2), (1000, 0.004), (100, 0.15), (30000, 0.02),
                                 (50, 0.8), (200, 0.5), (7, 1.0), (0, 0.3), (12, 0.0)])
def test_binomial_sampler_matches_the_binomial_law(n, p):
    from scipy import stats
    N = 1_000_000
    x = _draw(0, (n, p), N)
    assert x.min() >= 0 and x.max() <= n
    if p in (0.0, 1.0) or n == 0:
        assert (x == round(n * p)).all()
        return
    mean, var = n * p, n * p * (1 - p)
    assert abs(x.mean() - mean) < 5 * np.sqrt(var / N)
    assert abs(x.var() / var - 1) < 5 * np.sqrt(2.0 / N) + 1e-3
    # chi-square over the bins with expected count >= 20
    k = np.arange(n + 1)
    e = stats.binom.pmf(k, n, p) * N
    obs = np.bincount(x, minlength=n + 1)
    keep = e >= 20
    o2 = np.append(obs[keep], obs[~keep].sum())
    e2 = np.append(e[keep], e[~keep].sum())
    if e2[-1] < 20:
        o2, e2 = o2[:-1], e2[:-1]
        o2[-1] += obs[~keep].sum()
        e2[-1] += e[~keep].sum()
    chi2 = ((o2 - e2) ** 2 / e2).sum()
    pval = stats.chi2.sf(chi2, len(e2) - 1)
    assert pval > 1e-4, (chi2, len(e2), pval)


@pytest.mark.parametrize("k,mu,sigma,tau", [(1, 2.0, 0.5, 100.0), (20, 3.0, 1.0, 1768.0),
                                             (500, 1.5, 0.3, 1000.0), (10, 2.0, 0.5, 0.0),
                                             (3, 4.0, 0.0, 50.0)])
def test_first_time_sampler_is_the_minimum_of_k_arrivals(k, mu, sigma, tau):
    from scipy import stats
    N = 200_000
    x = _draw(1, (k, mu, sigma, tau), N)
    rng = np.random.default_rng(3)
    m = 40_000
    ref = (rng.exponential(tau, size=(m, k)) if tau > 0 else 0.0) + rng.normal(mu, sigma, size=(m, k))
    ref = ref.min(1)
    ks = stats.ks_2samp(x, ref)
    assert ks.pvalue > 1e-4, ks


def test_combine_matches_numpy():
    import torch
    import ctypes as C
    from crysplight_b200 import _lib
    from crysplight_b200.params import Readout
    rng = np.random.default_rng(1)
    K, n = 5, 1000
    raw = rng.standard_normal((K, n, 192)).astype(np.float32) * 0.05
    y_mean = np.concatenate([np.full(64, -5.0), np.full(64, 3.0), np.full(64, -0.5)]).astype(np.float32)
    y_std = np.concatenate([np.full(64, 0.8), np.full(64, 1.0), np.full(64, 0.2)]).astype(np.float32)
    raw[:, :10, :64] += rng.standard_normal((K, 10, 64)).astype(np.float32)   # disagreeing members
    xyz = (rng.uniform(0, 1, (n, 3)) * [48, 48, 22.4]).astype(np.float32)
    xyz[20] = [0.5, 24, 10]      # near a side face
    xyz[21] = [24, 24, 0.4]      # near the front face
    xyz[22] = [24, 24, 22.1]     # near the readout face: not wrapped
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
         dict(raw=raw, ym=y_mean, ys=y_std, xyz=xyz).items()}
    out = {k: torch.empty(s, dtype=t, device="cuda") for k, s, t in
           (("p", (n, 64), torch.float32), ("tm", (n, 64), torch.float32), ("ts", (n, 64), torch.float32),
            ("sp", (n,), torch.float32), ("fl", (n,), torch.uint8))}
    P = C.c_void_p
    rc = _lib.load().cl_surrogate_combine(
        P(d["raw"].data_ptr()), K, n, P(d["ym"].data_ptr()), P(d["ys"].data_ptr()), P(d["xyz"].data_ptr()),
        C.byref(BOX_BGO), C.byref(Readout(GRID)), 0.4, 0.02, 1.0, P(out["p"].data_ptr()),
        P(out["tm"].data_ptr()), P(out["ts"].data_ptr()), P(out["sp"].data_ptr()), P(out["fl"].data_ptr()), None)
    assert rc == 0
    torch.cuda.synchronize()
    o = {k: v.cpu().numpy() for k, v in out.items()}
    y = raw.astype(np.float64) * y_std + y_mean
    p = np.exp(y[:, :, :64])
    pm = p.mean(0)
    spread = p.std(0).sum(1) / pm.sum(1)
    assert np.allclose(o["p"], 0.4 * pm, rtol=1e-5)
    assert np.allclose(o["tm"], y[:, :, 64:128].mean(0), rtol=1e-5, atol=1e-5)
    assert np.allclose(o["ts"], np.exp(y[:, :, 128:].mean(0)), rtol=1e-5)
    assert np.allclose(o["sp"], spread, rtol=1e-4)
    d_wall = np.minimum.reduce([xyz[:, 0], 48 - xyz[:, 0], xyz[:, 1], 48 - xyz[:, 1], xyz[:, 2]])
    want = (spread > 0.02).astype(np.uint8) | ((d_wall < 1.0).astype(np.uint8) << 1)
    assert np.array_equal(o["fl"], want)
    assert o["fl"][20] & 2 and o["fl"][21] & 2 and not (o["fl"][22] & 2)
    assert (o["fl"][:10] & 1).all()


def _sites(n_points, photons, events_per_point, seed=3):
    pts = scan_points(n_points, BOX_BGO, seed=seed)
    xyz = np.repeat(pts, events_per_point, axis=0).astype(np.float32)
    n = xyz.shape[0]
    t0 = np.linspace(0.0, 0.2, n).astype(np.float32)
    ph = np.full(n, photons, np.int64)
    seg = np.arange(n, dtype=np.int32)
    return pts, xyz, t0, ph, seg


def _light_from_scan(engine, pts, photons, per_site_rows, pde):
    """Site light from a high-statistics scan (probabilities at PDE 1 times pde;
    transit-time mean and sigma from the exact moment sums)."""
    import torch
    from crysplight_b200 import _lib
    from crysplight_b200.fast_events import SiteLight
    from crysplight_b200.surrogate import scan_light
    scan = scan_light(engine, BOX_BGO, OP_BGO_ESR, GRID, points=pts, photons_per_point=photons, seed=77)
    c = np.maximum(scan.counts.astype(np.float64), 1)
    m1 = scan.tsum.astype(np.float64) / _lib.MOMENT_T_SCALE / c
    m2 = scan.tsum2.astype(np.float64) / _lib.MOMENT_T2_SCALE / c
    sig = np.sqrt(np.maximum(m2 - m1 * m1, 1e-6))
    p = scan.counts / photons * pde
    rep = lambda a: torch.from_numpy(np.repeat(a, per_site_rows, axis=0).astype(np.float32)).cuda()
    n = pts.shape[0] * per_site_rows
    return SiteLight(rep(p), rep(m1), rep(sig), torch.zeros(n, dtype=torch.float32, device="cuda"),
                     torch.zeros(n, dtype=torch.uint8, device="cuda")), scan


def test_all_fallback_equals_the_segment_transport(engine):
    """Every site flagged: the call is the plain Monte Carlo, bit for bit."""
    import torch
    from crysplight_b200.fast_events import SiteLight, sample_sites
    from crysplight_b200.params import OpticalParams
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, OP_BGO_ESR.sigma_alpha, 0.4)
    pts, xyz, t0, ph, seg = _sites(6, 3000, 4)
    n = xyz.shape[0]
    z = lambda *s: torch.zeros(*s, dtype=torch.float32, device="cuda")
    light = SiteLight(z(n, 64), z(n, 64), z(n, 64), z(n), torch.ones(n, dtype=torch.uint8, device="cuda"))
    T = lambda a: torch.from_numpy(a).cuda()
    (maps, tmin, npe, ctr, sampled), st = sample_sites(
        engine, BOX_BGO, op, GRID, TB80, xyz=T(xyz), t0=T(t0), photons=T(ph), segment=T(seg),
        n_segments=n, seed=99, tau_ns=TAU_BGO, light=light)
    ref = engine.run_segments(BOX_BGO, op, GRID, TB80, sources=xyz, photons_per_source=ph,
                              segment_of_source=seg, n_segments=n, seed=99, t0s=t0, tau_ns=TAU_BGO)
    m = maps.cpu().numpy().view(np.uint32).reshape(n, 64).T
    assert np.array_equal(m, ref.maps.reshape(64, n, order="F"))
    assert np.array_equal(tmin.cpu().numpy().reshape(n, 64).T.view(np.uint32),
                          ref.tmin.reshape(64, n, order="F").view(np.uint32))
    assert np.array_equal(npe.cpu().numpy(), ref.npe)
    assert st["fallback_sites"] == n and sampled.cpu().numpy().tolist() == [0, 0]


def test_sampling_reproduces_the_monte_carlo(engine):
    """Sites sampled from a high-statistics light response agree with the
    Monte Carlo of the same sites: summed SiPM counts within their Poisson
    errors, per-event chi2/ndf near its binomial expectation, and the mean
    first-hit time per SiPM within a few standard errors."""
    import torch
    from crysplight_b200.fast_events import compare_maps, sample_sites
    from crysplight_b200.params import OpticalParams
    op = OpticalParams(2.15, 1.45, 20000.0, 2222.0, 0.985, True, True, OP_BGO_ESR.sigma_alpha, 0.4)
    n_pts, per = 6, 300
    pts, xyz, t0, ph, seg = _sites(n_pts, 4000, per, seed=8)
    n = xyz.shape[0]
    light, scan = _light_from_scan(engine, pts, 8_000_000, per, 0.4)
    T = lambda a: torch.from_numpy(a).cuda()
    (maps, tmin, npe, ctr, sampled), st = sample_sites(
        engine, BOX_BGO, op, GRID, TB80, xyz=T(xyz), t0=T(t0), photons=T(ph), segment=T(seg),
        n_segments=n, seed=12, tau_ns=TAU_BGO, light=light)
    assert st["fallback_sites"] == 0
    s_maps = maps.cpu().numpy().view(np.uint32).reshape(n, 64).astype(np.int64)
    s_tmin = tmin.cpu().numpy().reshape(n, 64)
    assert int(sampled[0]) == int(ph.sum()) and int(sampled[1]) == int(s_maps.sum())
    assert np.array_equal(npe.cpu().numpy(), s_maps.sum(1))
    ref = engine.run_segments(BOX_BGO, op, GRID, TB80, sources=xyz, photons_per_source=ph,
                              segment_of_source=seg, n_segments=n, seed=5, t0s=t0, tau_ns=TAU_BGO)
    m_maps = ref.maps.reshape(64, n, order="F").T.astype(np.int64)
    m_tmin = ref.tmin.reshape(64, n, order="F").T
    for k in range(n_pts):
        sl = slice(k * per, (k + 1) * per)
        a, b = s_maps[sl].sum(0), m_maps[sl].sum(0)
        ok = b > 400
        z = (a[ok] - b[ok]) / np.sqrt(a[ok] + b[ok])
        assert np.abs(z).max() < 5.0, z
        assert abs(np.mean(z ** 2) - 1.0) < 0.6, np.mean(z ** 2)
    cmp = compare_maps(s_maps.T.reshape(8, 8, n), m_maps.T.reshape(8, 8, n))
    assert 0.8 < cmp["chi2_ndf_mean"] < 1.1, cmp
    # first-hit times of SiPMs hit in both: mean over events per (point, SiPM)
    for k in range(n_pts):
        sl = slice(k * per, (k + 1) * per)
        both = np.isfinite(s_tmin[sl]) & np.isfinite(m_tmin[sl])
        cols = both.sum(0) > 100
        for c in np.nonzero(cols)[0]:
            a = s_tmin[sl][both[:, c], c]
            b = m_tmin[sl][both[:, c], c]
            se = np.sqrt(a.var() / a.size + b.var() / b.size)
            assert abs(a.mean() - b.mean()) < 5 * se + 0.5, (k, c, a.mean(), b.mean(), se)


def test_depth_slab_expert_serves_the_sites_inside_its_slab(engine):
    """An expert ensemble replaces the main one exactly for the sites deeper
    than its slab start plus the margin; the other sites keep the main
    ensemble's outputs, and an expert spanning the whole crystal with the
    same networks changes nothing."""
    import os
    import torch
    from crysplight_b200.fast_events import SurrogateEvents
    from crysplight_b200.surrogate import LightSurrogate
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    main = LightSurrogate.load(os.path.join(root, "crysplight_b200", "surrogates", "bgo_esr.npz"))
    L = [float(v) for v in main.box_mm]
    rng = np.random.default_rng(4)
    xyz = np.stack([rng.uniform(0.5, L[0] - 0.5, 3000), rng.uniform(0.5, L[1] - 0.5, 3000),
                    rng.uniform(0.0, L[2], 3000)], 1).astype(np.float32)
    d = torch.from_numpy(xyz).cuda()
    from crysplight_b200.params import Readout, SipmGrid
    ro = Readout(SipmGrid(6.0, 8, 8))
    kw = dict(ro=ro, pde=0.4)

    def light(se):
        s = se.site_light(d, **kw)
        return {k: getattr(s, k).cpu().numpy() for k in ("p", "tmean", "tsig", "spread", "flag")}

    se0 = SurrogateEvents(main, engine)
    ref = light(se0)
    se0.close()
    whole = LightSurrogate(main.box_mm, main.y_mean, main.y_std, main.members, z_range=(0.0, L[2]),
                           first_pass=main.first_pass)
    se1 = SurrogateEvents(main, engine, experts=[whole], expert_margin_mm=1.0)
    same = light(se1)
    se1.close()
    for k in ref:
        assert np.array_equal(ref[k], same[k]), k
    # a slab over the readout half: its own input mapping, so other outputs
    z0 = 0.5 * L[2]
    slab = LightSurrogate(main.box_mm, main.y_mean, main.y_std, main.members[:3], z_range=(z0, L[2]),
                          first_pass=main.first_pass)
    se2 = SurrogateEvents(main, engine, experts=[slab], expert_margin_mm=1.0)
    mixed = light(se2)
    se2.close()
    inside = xyz[:, 2] >= z0 + 1.0
    se3 = SurrogateEvents(slab, engine)      # the slab ensemble alone, on the inside sites
    sub = se3.site_light(d[torch.from_numpy(np.nonzero(inside)[0]).cuda()], **kw)
    own = {k: getattr(sub, k).cpu().numpy() for k in ref}
    se3.close()
    assert 0 < inside.sum() < inside.size
    for k in ref:
        assert np.array_equal(mixed[k][~inside], ref[k][~inside]), k
        assert np.array_equal(mixed[k][inside], own[k]), k
    assert not np.array_equal(mixed["p"][inside], ref["p"][inside])
