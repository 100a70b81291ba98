"""Test infrastructure: a NumPy restatement of the surrogate's first-pass term
(``cl_surrogate_direct``), the checker of the CUDA kernel.

The first-pass probability of SiPM c for a photon emitted isotropically at
(x0, y0, z0): it reaches the readout face z = Lz (height h = Lz - z0) without
a bulk interaction, survival exp(-mu h / cos theta) with mu = 1/abs_len +
1/rayleigh (the reference's competition of the two exponential path lengths
against the wall distance, src/transport.jl:127-145), is transmitted by the
face (fresnel, src/optics.jl:10-19: unpolarised, total internal reflection
beyond the critical angle; the readout face interaction of
src/transport.jl:161-185) and lands in SiPM c's pixel
(src/transport.jl:96-108: ii = 1 + floor(x / pitch) clamped to nx).  Its
landing point lies on the circle of radius h tan(theta) about the site's
projection, uniform in azimuth, so

    D_c = 1/(4 pi) int (1 - R) exp(-mu h / cos theta) sin theta arc_c(theta) d theta

with arc_c the azimuth measure of the circle inside pixel c (exact) and the
polar integral by composite Gauss-Legendre quadrature.  ``sample`` is the
brute-force estimate of the same quantity (isotropic directions, straight to
the face).
"""
import numpy as np

TWO_PI = 2.0 * np.pi


def fresnel_R(n1, n2, cosi):
    q = n1 / n2
    sin2t = q * q * (1.0 - cosi * cosi)
    cost = np.sqrt(np.clip(1.0 - sin2t, 0.0, None))
    a = (n1 * cosi - n2 * cost) / (n1 * cosi + n2 * cost)
    b = (n1 * cost - n2 * cosi) / (n1 * cost + n2 * cosi)
    return np.where(sin2t >= 1.0, 1.0, 0.5 * (a * a + b * b))


def _x_intervals(a, b):
    a, b = np.clip(a, -1, 1), np.clip(b, -1, 1)
    aa, ab = np.arccos(a), np.arccos(b)
    return [(ab, aa), (TWO_PI - aa, TWO_PI - ab)]


def _y_intervals(a, b):
    a, b = np.clip(a, -1, 1), np.clip(b, -1, 1)
    ba, bb = np.arcsin(a), np.arcsin(b)
    neg = ba < 0
    split = neg & (bb >= 0)
    i1 = (np.where(neg, ba + TWO_PI, ba), np.where(neg, np.where(bb < 0, bb + TWO_PI, TWO_PI), bb))
    i2 = (np.zeros_like(ba), np.where(split, bb, 0.0))
    return [i1, i2, (np.pi - bb, np.pi - ba)]


def _overlap(i, j):
    return np.maximum(0.0, np.minimum(i[1], j[1]) - np.maximum(i[0], j[0]))


def direct(xyz, L, n1, n2, abs_len, rayleigh, pitch, nx, ny, panels=8, nodes=8):
    """(n, nx*ny) first-pass probabilities, Float64."""
    xyz = np.asarray(xyz, np.float64).reshape(-1, 3)
    mu = (0.0 if np.isinf(abs_len) else 1.0 / abs_len) + (0.0 if np.isinf(rayleigh) else 1.0 / rayleigh)
    out = np.zeros((xyz.shape[0], nx * ny))
    x0, y0 = xyz[:, 0], xyz[:, 1]
    h = L[2] - xyz[:, 2]
    inside = (h > 0) & (x0 >= 0) & (x0 <= L[0]) & (y0 >= 0) & (y0 <= L[1])
    h = np.where(inside, h, 1.0)
    th_max = np.arcsin(n2 / n1) if n2 < n1 else 0.5 * np.pi
    gx, gw = np.polynomial.legendre.leggauss(nodes)
    xe = [min(i * pitch, L[0]) for i in range(nx)] + [L[0]]
    ye = [min(j * pitch, L[1]) for j in range(ny)] + [L[1]]
    for p in range(panels):
        t0, t1 = th_max * p / panels, th_max * (p + 1) / panels
        for k in range(nodes):
            th = t0 + 0.5 * (t1 - t0) * (gx[k] + 1.0)
            c = np.cos(th)
            wt = 0.5 * (t1 - t0) * gw[k] * (1.0 - fresnel_R(n1, n2, c)) * np.exp(-mu * h / c) * np.sin(th)
            wt = np.where(inside, wt / (4.0 * np.pi), 0.0)
            rho = h * np.tan(th)
            for i in range(nx):
                xs = _x_intervals((xe[i] - x0) / rho, (xe[i + 1] - x0) / rho)
                for j in range(ny):
                    ys = _y_intervals((ye[j] - y0) / rho, (ye[j + 1] - y0) / rho)
                    out[:, j * nx + i] += wt * sum(_overlap(a, b) for a in xs for b in ys)
    return out


def sample(xyz1, L, n1, n2, abs_len, rayleigh, pitch, nx, ny, n=2_000_000, seed=1):
    """Brute-force estimate for one point: (nx*ny,) probabilities."""
    mu = (0.0 if np.isinf(abs_len) else 1.0 / abs_len) + (0.0 if np.isinf(rayleigh) else 1.0 / rayleigh)
    rng = np.random.default_rng(seed)
    uz = 1.0 - 2.0 * rng.random(n)
    ph = TWO_PI * rng.random(n)
    r = np.sqrt(1.0 - uz * uz)
    ux, uy = r * np.cos(ph), r * np.sin(ph)
    x0, y0, z0 = xyz1
    ok = uz > 0
    s = (L[2] - z0) / np.where(ok, uz, 1.0)
    xh, yh = x0 + s * ux, y0 + s * uy
    ok &= (xh >= 0) & (xh <= L[0]) & (yh >= 0) & (yh <= L[1])
    w = (1.0 - fresnel_R(n1, n2, np.where(ok, uz, 1.0))) * np.exp(-mu * s)
    i = np.minimum(np.floor(np.where(ok, xh, 0) / pitch).astype(int), nx - 1)
    j = np.minimum(np.floor(np.where(ok, yh, 0) / pitch).astype(int), ny - 1)
    out = np.zeros(nx * ny)
    np.add.at(out, (j * nx + i)[ok], w[ok])
    return out / n
