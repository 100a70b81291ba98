// cl_surrogate.cu — events from the learned light-response surrogate.
//
// The surrogate (cl_mlp.cu) maps an emission point to, per SiPM, the
// probability that a photon emitted there is detected by that SiPM and the
// mean and log standard deviation of the detected photons' transit times.
// For a 511 keV event the deposits ("sites") that the surrogate can be
// trusted with are sampled here instead of transported:
//
//   * surrogate_combine: the K ensemble members' outputs -> ensemble-mean
//     probabilities (times the PDE), transit-time mean and sigma, the members'
//     relative spread, and a fallback flag (spread above a threshold, the
//     site within a distance of a wrapped face, or detection probabilities
//     summing to 1 or more) that sends the site to the plain Monte Carlo;
//   * surrogate_sample: per unflagged site, the N emitted photons are split
//     over the SiPMs multinomially by a chain of conditional binomial draws
//     (n_j ~ Bin(N - sum_{i<j} n_i, p_j / (1 - sum_{i<j} p_i))), and each
//     SiPM's first-hit time is drawn exactly as the minimum of its n_j arrival
//     times, each an exponential emission delay (decay time tau) plus a
//     Gaussian transit time: the minimum's CDF is 1 - (1 - F)^n_j with F the
//     exponentially modified Gaussian CDF, inverted by safeguarded Newton.
//
// Binomial variates: inversion for n*p < 10, otherwise Hormann's BTRD
// (W. Hormann, "The generation of binomial random variates", J. Statist.
// Comput. Simul. 46 (1993) 101-110), both in Float64.  Uniforms come from
// Philox4x32-10 keyed with the event seed, counter (site lo, site hi, block,
// 0x53555247): a stream domain disjoint from the transport's photon streams
// (whose fourth counter word is 0).
//
// Every loop is bounded; a budget that runs out sets bit 2 of the error word
// and the site's remaining draws fall back to the mean.  A site whose segment
// id lies outside the maps is skipped and sets bit 3.
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/crysplight_cuda.h"
#include "cl_device.cuh"
#include "cl_surrogate.cuh"

namespace cl {
namespace sur {

constexpr uint32_t STREAM_TAG = 0x53555247u;   // "SURG": a site's binomial chain
constexpr uint32_t TIME_TAG = 0x53555254u;     // "SURT": a (site, SiPM) first-hit time
constexpr int CELLS = 64;                      // SiPMs of the readout grid
constexpr unsigned SAMPLER_BUDGET_BIT = 4u;

// Float64 uniforms in (0, 1) from one Philox stream.
struct Uni {
    uint32_t lo, hi, block, k0, k1;
    uint32_t buf[4];
    int left;
    __device__ void init(uint64_t stream, uint32_t key0, uint32_t key1)
    {
        lo = (uint32_t)stream; hi = (uint32_t)(stream >> 32); block = 0; k0 = key0; k1 = key1; left = 0;
    }
    __device__ double next()
    {
        if (left == 0) {
            const uint4 o = philox4x32_10(make_uint4(lo, hi, block, STREAM_TAG), k0, k1);
            block += 1u;
            buf[0] = o.x; buf[1] = o.y; buf[2] = o.z; buf[3] = o.w;
            left = 4;
        }
        const uint32_t x = buf[4 - left];
        left -= 1;
        return ((double)x + 0.5) * 0x1p-32;
    }
};

// Stirling-series remainder fc(k) = log(k!) - [(k + 1/2) log(k + 1) - (k + 1) + log(2 pi)/2].
__device__ double stirling_fc(int64_t k)
{
    const double N = (double)k + 1.0;
    if (k < 10) return lgamma(N) - (N - 0.5) * log(N) + N - 0.91893853320467274178;
    const double r = 1.0 / N, r2 = r * r;
    return (1.0 / 12.0 - (1.0 / 360.0 - (1.0 / 1260.0) * r2) * r2) * r;
}

// Inversion, n * p < 10, p <= 1/2 (sequential search from 0).
__device__ int64_t binom_inversion(int64_t n, double p, Uni& U, unsigned& bad)
{
    const double q = 1.0 - p, s = p / q, a = (double)(n + 1) * s;
    const double r0 = exp((double)n * log1p(-p));
    for (int attempt = 0; attempt < 64; ++attempt) {
        double u = U.next(), r = r0;
        int64_t x = 0;
        for (;;) {
            if (u <= r) return x;
            u -= r;
            ++x;
            if (x > n || x > 200) break;        // round-off tail: draw again
            r *= a / (double)x - s;
        }
    }
    bad |= SAMPLER_BUDGET_BIT;
    return (int64_t)((double)n * p + 0.5);
}

// BTRD, n * p >= 10, p <= 1/2.
__device__ int64_t binom_btrd(int64_t n, double p, Uni& U, unsigned& bad)
{
    const double q = 1.0 - p;
    const double np = (double)n * p, npq = np * q, spq = sqrt(npq);
    const int64_t m = (int64_t)floor((double)(n + 1) * p);
    const double r = p / q, nr = (double)(n + 1) * r;
    const double b = 1.15 + 2.53 * spq;
    const double a = -0.0873 + 0.0248 * b + 0.01 * p;
    const double c = np + 0.5;
    const double alpha = (2.83 + 5.1 / b) * spq;
    const double vr = 0.92 - 4.2 / b;
    const double urvr = 0.86 * vr;
    for (int it = 0; it < 1000; ++it) {
        double v = U.next(), u;
        if (v <= urvr) {
            u = v / vr - 0.43;
            return (int64_t)floor((2.0 * a / (0.5 - fabs(u)) + b) * u + c);
        }
        if (v >= vr) {
            u = U.next() - 0.5;
        } else {
            u = v / vr - 0.93;
            u = copysign(0.5, u) - u;
            v = U.next() * vr;
        }
        const double us = 0.5 - fabs(u);
        const double kd = floor((2.0 * a / us + b) * u + c);
        if (kd < 0.0 || kd > (double)n) continue;
        const int64_t k = (int64_t)kd;
        v = v * alpha / (a / (us * us) + b);
        const int64_t km = k > m ? k - m : m - k;
        if (km <= 15) {
            double f = 1.0;
            if (m < k) {
                for (int64_t i = m + 1; i <= k; ++i) f *= nr / (double)i - r;
            } else if (m > k) {
                for (int64_t i = k + 1; i <= m; ++i) v *= nr / (double)i - r;
            }
            if (v <= f) return k;
            continue;
        }
        v = log(v);
        const double kmd = (double)km;
        const double rho = (kmd / npq) * (((kmd / 3.0 + 0.625) * kmd + 1.0 / 6.0) / npq + 0.5);
        const double t = -kmd * kmd / (2.0 * npq);
        if (v < t - rho) return k;
        if (v > t + rho) continue;
        const double nm = (double)(n - m + 1);
        const double h = ((double)m + 0.5) * log(((double)m + 1.0) / (r * nm)) + stirling_fc(m) +
                         stirling_fc(n - m);
        const double nk = (double)(n - k + 1);
        if (v <= h + (double)(n + 1) * log(nm / nk) + ((double)k + 0.5) * log(nk * r / ((double)k + 1.0)) -
                     stirling_fc(k) - stirling_fc(n - k))
            return k;
    }
    bad |= SAMPLER_BUDGET_BIT;
    return (int64_t)(np + 0.5);
}

__device__ int64_t binomial(int64_t n, double p, Uni& U, unsigned& bad)
{
    if (n <= 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    const bool flip = p > 0.5;
    const double pp = flip ? 1.0 - p : p;
    const int64_t k = ((double)n * pp < 10.0) ? binom_inversion(n, pp, U, bad) : binom_btrd(n, pp, U, bad);
    return flip ? n - k : k;
}

// Exponentially modified Gaussian: X = E + T, E ~ Exp(rate lam), T ~ N(mu, sigma^2),
// in the standardised variable z = (t - mu) / sigma with ls = lam * sigma.
// Returns F(t) and sets *dens to the density f(t).
// Both terms carry exp(-z^2/2) where it would otherwise under/overflow
// (erfcx(x) = exp(x^2) erfc(x)).
__device__ double emg_cdf(double z, double ls, double lam, double* dens)
{
    constexpr double R2 = 0.70710678118654752440;
    const double w = z - ls;
    double phi_z, term2;
    if (w < 0.0) {
        term2 = 0.5 * exp(-0.5 * z * z) * erfcx(-w * R2);
    } else {
        term2 = 0.5 * exp(-ls * z + 0.5 * ls * ls) * erfc(-w * R2);
    }
    if (z < 0.0) phi_z = 0.5 * exp(-0.5 * z * z) * erfcx(-z * R2);
    else phi_z = 0.5 * erfc(-z * R2);
    *dens = lam * term2;            // density per unit t
    return phi_z - term2;
}

// Minimum of k >= 1 independent EMG(mu, sigma, tau) arrival times, by
// inverting P(min <= t) = 1 - (1 - F(t))^k at the uniform u in (0, 1).
__device__ double emg_min_u(int64_t k, double mu, double sigma, double tau, double u, unsigned& bad)
{
    const double lu = log(u) / (double)k;       // log of the survival level, < 0
    const double y = -expm1(lu);                // target F(t) in (0, 1)
    if (!(tau > 0.0)) return mu + sigma * normcdfinv(y);
    if (!(sigma > 0.0)) return mu - tau * lu;   // pure exponential: F = 1 - exp(-(t - mu)/tau)
    const double lam = 1.0 / tau, ls = lam * sigma;
    // bracket in z: F(lo) < y <= F(hi)
    double lo = -40.0, hi = 12.0 + (-tau * lu) / sigma + 0.5 * tau / sigma;
    double dens = 0.0;
    for (int g = 0; g < 64 && emg_cdf(hi, ls, lam, &dens) < y; ++g) hi = 2.0 * hi + 1.0;
    double z = fmin(fmax((-tau * lu) / sigma, lo), hi);
    for (int it = 0; it < 100; ++it) {
        const double F = emg_cdf(z, ls, lam, &dens) - y;
        if (F < 0.0) lo = z; else hi = z;
        const double fz = dens * sigma;            // dF/dz
        double zn = (fz > 0.0) ? z - F / fz : 0.5 * (lo + hi);
        if (!(zn > lo && zn < hi)) zn = 0.5 * (lo + hi);
        if (fabs(zn - z) < 1e-9 * fmax(1.0, fabs(z)) || hi - lo < 1e-9 * fmax(1.0, fabs(z)))
            return mu + sigma * zn;
        z = zn;
    }
    bad |= SAMPLER_BUDGET_BIT;
    return mu + sigma * z;
}

__device__ double emg_min(int64_t k, double mu, double sigma, double tau, Uni& U, unsigned& bad)
{
    return emg_min_u(k, mu, sigma, tau, U.next(), bad);
}

// The uniform of the first-hit time of SiPM c at site i: word 0 of its own
// Philox block (counter (site lo, site hi, c, "SURT")), disjoint from the
// site's binomial stream and from the transport's photon streams.
__device__ __forceinline__ double time_uniform(int64_t i, int c, uint32_t k0, uint32_t k1)
{
    const uint4 o = philox4x32_10(make_uint4((uint32_t)i, (uint32_t)((uint64_t)i >> 32), (uint32_t)c, TIME_TAG),
                                  k0, k1);
    return ((double)o.x + 0.5) * 0x1p-32;
}

// Warp-cooperative: each lane runs the binomial chain of one site (the
// chain is sequential over the SiPMs), recording the hit counts in shared
// memory; then the warp's lanes share out the first-hit times of all
// (site, SiPM) pairs that were hit, which cost far more than the chain (a
// safeguarded Newton inversion in Float64 each) and which thread-per-site
// code would leave to the lanes of the sites with the most hit SiPMs.  Each
// pair's time comes from its own uniform (time_uniform), so the result does
// not depend on which lane draws it.  Eight CTAs of 128 threads per SM
// (64 registers; the Float64 special functions' latency needs the warps more
// than the spilled registers cost).
constexpr int SAMPLE_WARPS = 4;
__global__ void __launch_bounds__(32 * SAMPLE_WARPS, 8) surrogate_sample(const SurSampleArgs A)
{
    __shared__ uint16_t s_k[SAMPLE_WARPS][CELLS][32];   // hit counts of the warp's sites, by SiPM
    __shared__ uint32_t s_mask[SAMPLE_WARPS][CELLS];    // lanes whose site hit the SiPM
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cells = A.cells;                          // <= CELLS (launcher)
    const int64_t nwarps = (int64_t)gridDim.x * SAMPLE_WARPS;
    unsigned bad = 0;
    unsigned long long ph = 0, det = 0;
    for (int64_t i0 = ((int64_t)blockIdx.x * SAMPLE_WARPS + wib) * 32; i0 < A.n; i0 += nwarps * 32) {
        // ---- the binomial chain of this lane's site ----
        const int64_t i = i0 + lane;
        int64_t left = 0, base = 0;
        if (i < A.n && !(A.flag && A.flag[i])) {
            left = A.photons[i];
            if (left > 0) {
                const int32_t sg = A.seg[i];
                if (sg < 0 || (int64_t)sg >= A.n_seg) { bad |= 8u; left = 0; }
                else { base = (int64_t)sg * cells; ph += (unsigned long long)left; }
            } else {
                left = 0;
            }
        }
        Uni U;
        U.init((uint64_t)i, A.k0, A.k1);
        const float* p = A.p + i * cells;
        double mass = 1.0;                          // probability not yet assigned
        for (int c = 0; c < cells; ++c) {
            int64_t k = 0;
            if (left > 0) {
                const double pc = (double)p[c];
                const double pcond = mass > 0.0 ? fmin(fmax(pc / mass, 0.0), 1.0) : 1.0;
                mass -= pc;
                k = binomial(left, pcond, U, bad);
                if (k > 0) {
                    left -= k;
                    det += (unsigned long long)k;
                    atomicAdd(A.maps + base + c, (uint32_t)k);
                    if (k > 65535) {
                        // beyond the shared counts' range: this lane draws its time now
                        const double t = emg_min_u(k, (double)A.tmean[i * cells + c], (double)A.tsig[i * cells + c],
                                                   (double)A.tau, time_uniform(i, c, A.k0, A.k1), bad);
                        atomicMin(A.keys + base + c, float_key((float)((double)A.t0[i] + t)));
                        k = 0;
                    }
                }
            }
            s_k[wib][c][lane] = (uint16_t)k;
            const unsigned m = __ballot_sync(0xffffffffu, k > 0);
            if (lane == 0) s_mask[wib][c] = m;
        }
        __syncwarp();
        // ---- the first-hit times of every (site, SiPM) pair hit, shared out ----
        int total = 0;
        for (int c = 0; c < cells; ++c) total += __popc(s_mask[wib][c]);
        int c = 0, before = 0;                      // items of SiPMs < c
        for (int item = lane; item < total; item += 32) {
            while (item >= before + __popc(s_mask[wib][c])) { before += __popc(s_mask[wib][c]); ++c; }
            const unsigned m = s_mask[wib][c];
            const int sl = (int)__fns(m, 0u, item - before + 1);     // the site's lane
            const int64_t is = i0 + sl;
            const int64_t kk = s_k[wib][c][sl];
            const double t = emg_min_u(kk, (double)A.tmean[is * cells + c], (double)A.tsig[is * cells + c],
                                       (double)A.tau, time_uniform(is, c, A.k0, A.k1), bad);
            atomicMin(A.keys + (int64_t)A.seg[is] * cells + c, float_key((float)((double)A.t0[is] + t)));
        }
        __syncwarp();
    }
    if (A.stats) {
        // one pair of atomics per warp
        for (int o = 16; o > 0; o >>= 1) {
            ph += __shfl_down_sync(0xffffffffu, ph, o);
            det += __shfl_down_sync(0xffffffffu, det, o);
        }
        if ((threadIdx.x & 31) == 0 && (ph | det)) {
            atomicAdd(A.stats, ph);
            atomicAdd(A.stats + 1, det);
        }
    }
    if (bad) atomicOr(A.err, bad);
}

// Ensemble reduction: 64 threads per site (one per SiPM), 4 sites per CTA.
struct CombineArgs {
    const float* raw;        // [K][n][3 * cells] standardised member outputs
    int32_t K;
    int64_t n;
    const float* y_mean;     // [3 * cells]
    const float* y_std;      // [3 * cells]
    const float* xyz;        // [n][3] mm
    const float* direct;     // [n][CELLS] first-pass probabilities added to the members' (may be null)
    float L0, L1, L2;
    int32_t front_wrapped;
    float pde, spread_max, wall_min_mm;
    float* p;
    float* tmean;
    float* tsig;
    float* spread;
    uint8_t* flag;
};

constexpr int SITES_PER_CTA = 4;

__global__ void __launch_bounds__(CELLS * SITES_PER_CTA) surrogate_combine(const CombineArgs A)
{
    __shared__ double red[SITES_PER_CTA][2][2];
    const int c = threadIdx.x % CELLS;
    const int s_loc = threadIdx.x / CELLS;
    const int warp_in_site = c / 32;
    const float mp = A.y_mean[c], sp = A.y_std[c];
    const float mt = A.y_mean[CELLS + c], st = A.y_std[CELLS + c];
    const float ml = A.y_mean[2 * CELLS + c], sl = A.y_std[2 * CELLS + c];
    for (int64_t s0 = (int64_t)blockIdx.x * SITES_PER_CTA; s0 < A.n; s0 += (int64_t)gridDim.x * SITES_PER_CTA) {
        const int64_t i = s0 + s_loc;
        double sum_p = 0.0, sum_p2 = 0.0, sum_t = 0.0, sum_l = 0.0;
        if (i < A.n) {
            for (int k = 0; k < A.K; ++k) {
                const float* row = A.raw + ((int64_t)k * A.n + i) * (3 * CELLS);
                const double pk = exp((double)row[c] * sp + mp);
                sum_p += pk;
                sum_p2 += pk * pk;
                sum_t += (double)row[CELLS + c] * st + mt;
                sum_l += (double)row[2 * CELLS + c] * sl + ml;
            }
        }
        const double invK = 1.0 / (double)A.K;
        const double pr = sum_p * invK;
        const double var = fmax(sum_p2 * invK - pr * pr, 0.0);
        // the first-pass term is the same for every member: it adds to the
        // mean and to the total the spread is relative to, not to the spread
        const double pm = pr + (A.direct && i < A.n ? (double)A.direct[i * CELLS + c] : 0.0);
        double a = sqrt(var), b = pm;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if ((c & 31) == 0) { red[s_loc][warp_in_site][0] = a; red[s_loc][warp_in_site][1] = b; }
        __syncthreads();
        if (i < A.n) {
            A.p[i * CELLS + c] = (float)(pm * (double)A.pde);
            A.tmean[i * CELLS + c] = (float)(sum_t * invK);
            A.tsig[i * CELLS + c] = (float)exp(sum_l * invK);
            if (c == 0) {
                const double num = red[s_loc][0][0] + red[s_loc][1][0];
                const double den = red[s_loc][0][1] + red[s_loc][1][1];
                const float spr = (float)(num / fmax(den, 1e-30));
                const float x = A.xyz[3 * i], y = A.xyz[3 * i + 1], z = A.xyz[3 * i + 2];
                float d = fminf(fminf(x, A.L0 - x), fminf(y, A.L1 - y));
                if (A.front_wrapped) d = fminf(d, z);
                uint8_t f = 0;
                if (!(spr <= A.spread_max)) f |= 1u;
                if (d < A.wall_min_mm) f |= 2u;
                if (!(den * (double)A.pde < 0.999)) f |= 4u;   // not a probability split: Monte Carlo
                A.spread[i] = spr;
                A.flag[i] = f;
            }
        }
        __syncthreads();
    }
}

// First-pass light (the analytic part of the light response): the
// probability that a photon emitted isotropically at a site reaches the
// readout face z = Lz without a bulk interaction and crosses into SiPM c
// there, at PDE 1.  A photon leaving at polar angle theta from the face normal
// travels h / cos(theta) (h = Lz - z) and survives absorption and Rayleigh
// scattering with probability exp(-mu h / cos theta), mu = 1/abs_len +
// 1/rayleigh (the competition of the two exponential path lengths against
// the face distance); the face transmits it with probability 1 - R(cos
// theta) (the same Fresnel coefficients, total internal reflection beyond
// the critical angle); it lands on the circle of radius rho = h tan(theta)
// about the site's projection, uniformly in azimuth, and is detected by the
// SiPM whose pixel contains the landing point (pixel c = j nx + i for
// floor(x / pitch) = i, the last column and row reaching the face edge;
// landing points off the face belong to a side wall first and are not
// first-pass light).  So
//     D_c = 1/(4 pi) int_0^theta_max (1 - R) exp(-mu h / cos theta) sin theta
//           * (arc of the circle inside pixel c) d theta,
// with the arcs exact (intersections of the circle with the pixel's column
// and row strips) and theta by composite Gauss-Legendre quadrature (8 panels
// of 8 nodes up to the critical angle; 64 threads per site, one per node).
// The nodes' contributions are summed as 2^-40 fixed-point integers, so the
// result does not depend on the order the threads add them in: a site's
// term is the same bits in any batch.
// The rest of the light response (reflections, scattering) varies slowly
// over the SiPM plane; a surrogate trained on it learns what the first-pass
// term's sharp pixel edges would otherwise ask of it.
namespace {
// 8-point Gauss-Legendre nodes and weights on [-1, 1] (positive half)
__constant__ double c_gl_x[4] = {0.1834346424956498, 0.5255324099163290, 0.7966664774136267, 0.9602898564975363};
__constant__ double c_gl_w[4] = {0.3626837833783620, 0.3137066458778873, 0.2223810344533745, 0.1012285362903763};
}

struct DirectArgs {
    const float* xyz;        // [n][3] mm
    int64_t n;
    float L0, L1, L2;
    float n1, n2, mu;        // crystal and coupling indices, attenuation 1/mm
    float pitch;
    int32_t nx, ny;
    float* out;              // [n][CELLS]
};

constexpr int DIRECT_NODES = 64;
constexpr double DIRECT_FIX = 1099511627776.0;   // 2^40
constexpr int DIRECT_SITES_PER_CTA = 4;
constexpr float TWO_PI_ARC = 6.283185307179586f;

// Length in [0, 2pi) of the circle's azimuths phi with cos(phi) in [ca, cb]
// and sin(phi) in [sa, sb] (bounds clamped to [-1, 1]).
__device__ __forceinline__ float arc_in_box(float ca, float cb, float sa, float sb)
{
    ca = fminf(fmaxf(ca, -1.0f), 1.0f); cb = fminf(fmaxf(cb, -1.0f), 1.0f);
    sa = fminf(fmaxf(sa, -1.0f), 1.0f); sb = fminf(fmaxf(sb, -1.0f), 1.0f);
    const float aa = acosf(ca), ab = acosf(cb);          // ab <= aa
    const float x1l = ab, x1h = aa, x2l = TWO_PI_ARC - aa, x2h = TWO_PI_ARC - ab;
    const float ba = asinf(sa), bb = asinf(sb);          // in [-pi/2, pi/2]
    float y1l, y1h, y2l = 0.0f, y2h = 0.0f;
    if (ba >= 0.0f) { y1l = ba; y1h = bb; }
    else if (bb < 0.0f) { y1l = ba + TWO_PI_ARC; y1h = bb + TWO_PI_ARC; }
    else { y1l = ba + TWO_PI_ARC; y1h = TWO_PI_ARC; y2h = bb; }
    const float pi = 0.5f * TWO_PI_ARC;
    const float y3l = pi - bb, y3h = pi - ba;
    float arc = 0.0f;
    arc += fmaxf(0.0f, fminf(x1h, y1h) - fmaxf(x1l, y1l));
    arc += fmaxf(0.0f, fminf(x1h, y2h) - fmaxf(x1l, y2l));
    arc += fmaxf(0.0f, fminf(x1h, y3h) - fmaxf(x1l, y3l));
    arc += fmaxf(0.0f, fminf(x2h, y1h) - fmaxf(x2l, y1l));
    arc += fmaxf(0.0f, fminf(x2h, y2h) - fmaxf(x2l, y2l));
    arc += fmaxf(0.0f, fminf(x2h, y3h) - fmaxf(x2l, y3l));
    return arc;
}

__global__ void __launch_bounds__(DIRECT_NODES * DIRECT_SITES_PER_CTA) surrogate_direct(const DirectArgs A)
{
    __shared__ unsigned long long acc[DIRECT_SITES_PER_CTA][CELLS];
    const int q = threadIdx.x % DIRECT_NODES;
    const int s_loc = threadIdx.x / DIRECT_NODES;
    // this thread's quadrature node: panel q / 8, node q % 8 (mirror pairs)
    const int panel = q / 8, k = q % 8;
    const double gx = k < 4 ? -c_gl_x[3 - k] : c_gl_x[k - 4];
    const double gw = k < 4 ? c_gl_w[3 - k] : c_gl_w[k - 4];
    const double n1 = A.n1, n2 = A.n2;
    const double th_max = n2 < n1 ? asin(n2 / n1) : 0.5 * 3.141592653589793;
    const double t0 = th_max * panel / 8.0, t1 = th_max * (panel + 1) / 8.0;
    const double th = t0 + 0.5 * (t1 - t0) * (gx + 1.0);
    const double c = cos(th), sn = sin(th);
    // Fresnel transmission at the readout face (as fresnel_q2, in Float64)
    double T = 0.0;
    {
        const double q2 = (n1 / n2) * (n1 / n2);
        const double sin2t = q2 * (1.0 - c * c);
        if (sin2t < 1.0) {
            const double ct = sqrt(1.0 - sin2t);
            const double a = (n1 * c - n2 * ct) / (n1 * c + n2 * ct);
            const double b = (n1 * ct - n2 * c) / (n1 * ct + n2 * c);
            T = 1.0 - 0.5 * (a * a + b * b);
        }
    }
    const double w_node = 0.5 * (t1 - t0) * gw * T * sn / (4.0 * 3.141592653589793);
    const float tan_th = (float)(sn / c);
    for (int64_t s0 = (int64_t)blockIdx.x * DIRECT_SITES_PER_CTA; s0 < A.n; s0 += (int64_t)gridDim.x * DIRECT_SITES_PER_CTA) {
        const int64_t i = s0 + s_loc;
        for (int t = threadIdx.x; t < DIRECT_SITES_PER_CTA * CELLS; t += blockDim.x) (&acc[0][0])[t] = 0ull;
        __syncthreads();
        if (i < A.n) {
            const float x0 = A.xyz[3 * i], y0 = A.xyz[3 * i + 1], z0 = A.xyz[3 * i + 2];
            const float h = A.L2 - z0;
            if (h > 0.0f && x0 >= 0.0f && x0 <= A.L0 && y0 >= 0.0f && y0 <= A.L1) {
                const float wt = (float)(w_node * exp(-(double)A.mu * (double)h / c));
                const float rho = h * tan_th;
                const float inv = 1.0f / rho;
                int ilo = (int)floorf((x0 - rho) / A.pitch), ihi = (int)floorf((x0 + rho) / A.pitch);
                int jlo = (int)floorf((y0 - rho) / A.pitch), jhi = (int)floorf((y0 + rho) / A.pitch);
                ilo = max(ilo, 0); jlo = max(jlo, 0); ihi = min(ihi, A.nx - 1); jhi = min(jhi, A.ny - 1);
                for (int jj = jlo; jj <= jhi; ++jj) {
                    const float ya = fminf(jj * A.pitch, A.L1);
                    const float yb = jj == A.ny - 1 ? A.L1 : fminf((jj + 1) * A.pitch, A.L1);
                    for (int ii = ilo; ii <= ihi; ++ii) {
                        const float xa = fminf(ii * A.pitch, A.L0);
                        const float xb = ii == A.nx - 1 ? A.L0 : fminf((ii + 1) * A.pitch, A.L0);
                        const float arc = arc_in_box((xa - x0) * inv, (xb - x0) * inv, (ya - y0) * inv,
                                                     (yb - y0) * inv);
                        if (arc > 0.0f)
                            atomicAdd(&acc[s_loc][jj * A.nx + ii],
                                      __double2ull_rn((double)wt * (double)arc * DIRECT_FIX));
                    }
                }
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < DIRECT_SITES_PER_CTA * CELLS; t += blockDim.x) {
            const int64_t site = s0 + t / CELLS;
            if (site < A.n) A.out[site * CELLS + t % CELLS] = (float)((double)(&acc[0][0])[t] / DIRECT_FIX);
        }
        __syncthreads();
    }
}

// Network inputs of the sites: x, y scaled to [-1, 1] and the depth through
// w(t) = (1 - a) t + a (1 - sqrt(1 - t)), t = z / Lz clamped to [0, 1].
__global__ void surrogate_inputs(const float* __restrict__ xyz, int64_t n, float L0, float L1, float L2,
                                 float a, float* __restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        const float t = fminf(fmaxf(z / L2, 0.0f), 1.0f);
        const float w = (1.0f - a) * t + a * (1.0f - sqrtf(1.0f - t));
        out[3 * i] = 2.0f * x / L0 - 1.0f;
        out[3 * i + 1] = 2.0f * y / L1 - 1.0f;
        out[3 * i + 2] = 2.0f * w - 1.0f;
    }
}

// Diagnostics: fn 0 = binomial(n = par[0], p = par[1]) -> int64,
// fn 1 = emg_min(k = par[0], mu = par[1], sigma = par[2], tau = par[3]) -> double.
__global__ void debug_sampler(int fn, double p0, double p1, double p2, double p3, int64_t n,
                              uint32_t k0, uint32_t k1, void* out, unsigned int* err)
{
    unsigned bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        Uni U;
        U.init((uint64_t)i, k0, k1);
        if (fn == 0) ((int64_t*)out)[i] = binomial((int64_t)p0, p1, U, bad);
        else ((double*)out)[i] = emg_min((int64_t)p0, p1, p2, p3, U, bad);
    }
    if (bad && err) atomicOr(err, bad);
}

}  // namespace sur

cudaError_t launch_surrogate_sample(const SurSampleArgs& a, int num_sms, cudaStream_t st)
{
    if (a.n <= 0) return cudaSuccess;
    if (a.cells < 1 || a.cells > sur::CELLS) return cudaErrorInvalidValue;
    const int64_t want = (a.n + 32 * sur::SAMPLE_WARPS - 1) / (32 * sur::SAMPLE_WARPS);
    const int64_t cap = (int64_t)num_sms * 16;
    sur::surrogate_sample<<<(unsigned)(want < cap ? want : cap), 32 * sur::SAMPLE_WARPS, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cl

extern "C" {

int cl_surrogate_combine(const float* d_raw, int32_t members, int64_t n_sites,
                         const float* d_y_mean, const float* d_y_std, const float* d_xyz,
                         const cl_box* box, const cl_readout* ro, float pde,
                         float spread_max, float wall_min_mm,
                         float* d_p, float* d_tmean, float* d_tsig, float* d_spread,
                         uint8_t* d_flag, void* stream)
{
    return cl_surrogate_combine_direct(d_raw, members, n_sites, d_y_mean, d_y_std, d_xyz, nullptr, box, ro, pde,
                                       spread_max, wall_min_mm, d_p, d_tmean, d_tsig, d_spread, d_flag, stream);
}

int cl_surrogate_combine_direct(const float* d_raw, int32_t members, int64_t n_sites,
                                const float* d_y_mean, const float* d_y_std, const float* d_xyz,
                                const float* d_direct, const cl_box* box, const cl_readout* ro, float pde,
                                float spread_max, float wall_min_mm,
                                float* d_p, float* d_tmean, float* d_tsig, float* d_spread,
                                uint8_t* d_flag, void* stream)
{
    if (!box || !ro || members < 1 || n_sites < 0) return CL_ERR_ARG;
    if ((int64_t)ro->grid.nx * ro->grid.ny != cl::sur::CELLS) return CL_ERR_ARG;
    if (n_sites == 0) return CL_OK;
    if (!d_raw || !d_y_mean || !d_y_std || !d_xyz || !d_p || !d_tmean || !d_tsig || !d_spread || !d_flag)
        return CL_ERR_ARG;
    if (!(pde >= 0.0f && pde <= 1.0f)) return CL_ERR_ARG;
    cl::sur::CombineArgs a;
    a.raw = d_raw; a.K = members; a.n = n_sites; a.y_mean = d_y_mean; a.y_std = d_y_std; a.xyz = d_xyz;
    a.direct = d_direct;
    a.L0 = box->L[0]; a.L1 = box->L[1]; a.L2 = box->L[2];
    a.front_wrapped = ro->two_sided ? 0 : 1;
    a.pde = pde; a.spread_max = spread_max; a.wall_min_mm = wall_min_mm;
    a.p = d_p; a.tmean = d_tmean; a.tsig = d_tsig; a.spread = d_spread; a.flag = d_flag;
    const int64_t want = (n_sites + cl::sur::SITES_PER_CTA - 1) / cl::sur::SITES_PER_CTA;
    const unsigned grid = (unsigned)(want < 148 * 64 ? want : 148 * 64);
    cl::sur::surrogate_combine<<<grid, cl::sur::CELLS * cl::sur::SITES_PER_CTA, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

int cl_surrogate_direct(const float* d_xyz, int64_t n_sites, const cl_box* box, const cl_optical_params* op,
                        const cl_readout* ro, float* d_out, void* stream)
{
    if (!box || !op || !ro || n_sites < 0) return CL_ERR_ARG;
    if ((int64_t)ro->grid.nx * ro->grid.ny != cl::sur::CELLS || ro->grid.nx < 1 || !(ro->grid.pitch_mm > 0.0f))
        return CL_ERR_ARG;
    // the model: one full readout face at z = Lz
    if (ro->disc || ro->two_sided) return CL_ERR_ARG;
    if (!(op->n_crystal > 0.0f) || !(op->n_coupling > 0.0f) || !(op->abs_len_mm > 0.0f) || !(op->rayleigh_mm > 0.0f))
        return CL_ERR_ARG;
    if (n_sites == 0) return CL_OK;
    if (!d_xyz || !d_out) return CL_ERR_ARG;
    cl::sur::DirectArgs a;
    a.xyz = d_xyz; a.n = n_sites; a.L0 = box->L[0]; a.L1 = box->L[1]; a.L2 = box->L[2];
    a.n1 = op->n_crystal; a.n2 = op->n_coupling;
    a.mu = (float)((std::isinf(op->abs_len_mm) ? 0.0 : 1.0 / (double)op->abs_len_mm) +
                   (std::isinf(op->rayleigh_mm) ? 0.0 : 1.0 / (double)op->rayleigh_mm));
    a.pitch = ro->grid.pitch_mm; a.nx = ro->grid.nx; a.ny = ro->grid.ny; a.out = d_out;
    const int64_t want = (n_sites + cl::sur::DIRECT_SITES_PER_CTA - 1) / cl::sur::DIRECT_SITES_PER_CTA;
    const unsigned grid = (unsigned)(want < 148 * 32 ? want : 148 * 32);
    cl::sur::surrogate_direct<<<grid, cl::sur::DIRECT_NODES * cl::sur::DIRECT_SITES_PER_CTA, 0,
                                (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

int cl_surrogate_inputs(const float* d_xyz, int64_t n_sites, const cl_box* box, float z_warp, float* d_out,
                        void* stream)
{
    if (!box || n_sites < 0 || !(z_warp >= 0.0f && z_warp <= 1.0f)) return CL_ERR_ARG;
    if (n_sites == 0) return CL_OK;
    if (!d_xyz || !d_out) return CL_ERR_ARG;
    const int64_t want = (n_sites + 255) / 256;
    const unsigned grid = (unsigned)(want < 148 * 32 ? want : 148 * 32);
    cl::sur::surrogate_inputs<<<grid, 256, 0, (cudaStream_t)stream>>>(d_xyz, n_sites, box->L[0], box->L[1],
                                                                      box->L[2], z_warp, d_out);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

int cl_debug_sampler(int fn, const double* par, int64_t n, uint64_t seed, void* d_out,
                     unsigned int* d_err, void* stream)
{
    if ((fn != 0 && fn != 1) || !par || n < 0 || (n > 0 && !d_out)) return CL_ERR_ARG;
    if (n == 0) return CL_OK;
    const unsigned grid = (unsigned)((n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16);
    cl::sur::debug_sampler<<<grid, 256, 0, (cudaStream_t)stream>>>(fn, par[0], par[1], par[2], par[3], n,
                                                                   (uint32_t)seed, (uint32_t)(seed >> 32),
                                                                   d_out, d_err);
    return cudaGetLastError() == cudaSuccess ? CL_OK : CL_ERR_CUDA;
}

}  // extern "C"
