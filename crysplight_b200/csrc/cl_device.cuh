// cl_device.cuh — device-side building blocks of the transport engine:
// Philox4x32-10 streams, Float32 elementary functions, and the per-photon
// physics of one bounce-loop iteration.
//
// Arithmetic contract (what makes results identical to the reference's CPU
// transport, src/transport.jl):
//   * compiled with --fmad=false: no multiply-add contraction, every float
//     operation rounds once as in Julia;
//   * IEEE division and square root (no fast-math);
//   * log/sin/cos of Float32 arguments are evaluated in Float64 and rounded
//     once to Float32 (see cl_logf / cl_sincosf);
//   * expressions keep the reference's association and draw order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cl_tables.h"

namespace cl {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11), as keyed in src/philox.jl:5-28.
// ---------------------------------------------------------------------------
constexpr uint32_t PHILOX_M0 = 0xD2511F53u;
constexpr uint32_t PHILOX_M1 = 0xCD9E8D57u;
constexpr uint32_t PHILOX_W0 = 0x9E3779B9u;
constexpr uint32_t PHILOX_W1 = 0xBB67AE85u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)PHILOX_M0 * c.x;   // IMAD.WIDE.U32
        const uint64_t p1 = (uint64_t)PHILOX_M1 * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    return c;
}

// A photon's uniform stream (PhiloxStream / PhiloxState, src/philox.jl:34-62,
// src/kernel.jl:15-46).  Key = seed, counter = (pid lo, pid hi, block, 0).
// Up to eight outputs (two blocks) are buffered; draw() pops in order, so the
// sequence is the reference's regardless of when blocks are generated.
struct Stream {
    uint32_t pid_lo, pid_hi, block;
    uint32_t b0, b1, b2, b3, b4, b5, b6, b7;
    int n;  // buffered outputs
};

__device__ __forceinline__ void stream_init(Stream& s, uint64_t pid)
{
    s.pid_lo = (uint32_t)pid;
    s.pid_hi = (uint32_t)(pid >> 32);
    s.block = 0;
    s.n = 0;
    s.b0 = s.b1 = s.b2 = s.b3 = s.b4 = s.b5 = s.b6 = s.b7 = 0;
}

// Append one block behind the buffered outputs (requires n <= 4).
__device__ __forceinline__ void stream_fill(Stream& s, uint32_t k0, uint32_t k1)
{
    const uint4 o = philox4x32_10(make_uint4(s.pid_lo, s.pid_hi, s.block, 0u), k0, k1);
    s.block += 1u;
    if (s.n == 0) {
        s.b0 = o.x; s.b1 = o.y; s.b2 = o.z; s.b3 = o.w;
    } else {
        // n in 1..4: place after the n buffered outputs
        if (s.n == 1) { s.b1 = o.x; s.b2 = o.y; s.b3 = o.z; s.b4 = o.w; }
        else if (s.n == 2) { s.b2 = o.x; s.b3 = o.y; s.b4 = o.z; s.b5 = o.w; }
        else if (s.n == 3) { s.b3 = o.x; s.b4 = o.y; s.b5 = o.z; s.b6 = o.w; }
        else { s.b4 = o.x; s.b5 = o.y; s.b6 = o.z; s.b7 = o.w; }
    }
    s.n += 4;
}

// Top the buffer up to at least 5 outputs; called at convergent points so
// the Philox rounds execute once for the whole warp.
__device__ __forceinline__ void stream_topup(Stream& s, uint32_t k0, uint32_t k1)
{
    if (s.n <= 4) stream_fill(s, k0, k1);
}

__device__ __forceinline__ uint32_t stream_next(Stream& s, uint32_t k0, uint32_t k1)
{
    if (s.n == 0) stream_fill(s, k0, k1);
    const uint32_t x = s.b0;
    s.b0 = s.b1; s.b1 = s.b2; s.b2 = s.b3; s.b3 = s.b4;
    s.b4 = s.b5; s.b5 = s.b6; s.b6 = s.b7;
    s.n -= 1;
    return x;
}

// randu, src/philox.jl:62: ((x >>> 8) + 1.0f0) * 2^-24, exact, in (0, 1].
__device__ __forceinline__ float randu(Stream& s, uint32_t k0, uint32_t k1)
{
    const uint32_t x = stream_next(s, k0, k1);
    return __fmul_rn(__fadd_rn((float)(x >> 8), 1.0f), 0x1p-24f);
}

// ---------------------------------------------------------------------------
// Float32 elementary functions.  Each is evaluated in Float64 to about 2^-51
// relative error and rounded once, so it returns the correctly rounded
// Float32 except when the exact value lies within ~2^-51 of a rounding
// boundary.  Arguments outside the transport's domain take a slow path
// through the CUDA double-precision library functions.
// ---------------------------------------------------------------------------

// Natural log.  Table-driven (Tang 1990): x = 2^e * m, m in [sqrt(1/2), sqrt(2)),
// m = F_j (1 + r) with F_j = 1 + j/64, ln x = e ln2 + ln F_j + log1p(r),
// |r| < 1/90, log1p by its Taylor series to r^8.
__device__ __forceinline__ float cl_logf(float x, const double2* __restrict__ tab)
{
    const uint32_t b = __float_as_uint(x);
    if (b - 0x00800000u >= 0x7f000000u)       // not a positive normal finite float
        return __double2float_rn(log((double)x));
    int e = (int)(b >> 23) - 127;
    uint32_t mb = b & 0x007fffffu;
    const int hi = mb >= 0x3504f3u;          // m >= sqrt(2): use m/2, e+1
    e += hi;
    mb |= hi ? 0x3f000000u : 0x3f800000u;
    const double m = (double)__uint_as_float(mb);
    const int j = __double2int_rn((m - 1.0) * 64.0);
    const double F = 1.0 + (double)j * 0.015625;
    const double2 t = tab[j - CLM_LOG_JMIN];
    const double r = (m - F) * t.x;            // m - F is exact
    double p = CLM_L8;
    p = fma(p, r, CLM_L7);
    p = fma(p, r, CLM_L6);
    p = fma(p, r, CLM_L5);
    p = fma(p, r, CLM_L4);
    p = fma(p, r, CLM_L3);
    p = fma(p, r, CLM_L2);
    const double lp = fma(p * r, r, r);        // log1p(r)
    const double res = fma((double)e, CLM_LN2, t.y) + lp;
    return __double2float_rn(res);
}

// sin and cos together.  Cody-Waite reduction x = q pi/2 + r with a two-term
// pi/2, |r| <= pi/4, then Taylor polynomials (sin to r^17, cos to r^16).
__device__ __forceinline__ void cl_sincosf(float x, float* sp, float* cp)
{
    const double xd = (double)x;
    if (!(fabs(xd) <= 1.0e4)) {
        *sp = __double2float_rn(sin(xd));
        *cp = __double2float_rn(cos(xd));
        return;
    }
    if (xd == 0.0) {                           // sin(+-0) = +-0, cos(+-0) = 1
        *sp = x;
        *cp = 1.0f;
        return;
    }
    const double q = rint(xd * CLM_2_OVER_PI);
    double r = fma(-q, CLM_PIO2_HI, xd);
    r = fma(-q, CLM_PIO2_LO, r);
    const double r2 = r * r;
    double ps = CLM_S17;
    ps = fma(ps, r2, CLM_S15);
    ps = fma(ps, r2, CLM_S13);
    ps = fma(ps, r2, CLM_S11);
    ps = fma(ps, r2, CLM_S9);
    ps = fma(ps, r2, CLM_S7);
    ps = fma(ps, r2, CLM_S5);
    ps = fma(ps, r2, CLM_S3);
    const double sn = fma(r * r2, ps, r);
    double pc = CLM_C16;
    pc = fma(pc, r2, CLM_C14);
    pc = fma(pc, r2, CLM_C12);
    pc = fma(pc, r2, CLM_C10);
    pc = fma(pc, r2, CLM_C8);
    pc = fma(pc, r2, CLM_C6);
    pc = fma(pc, r2, CLM_C4);
    pc = fma(pc, r2, CLM_C2);
    const double cs = fma(r2, pc, 1.0);
    const int iq = (int)q;
    double s = (iq & 1) ? cs : sn;
    double c = (iq & 1) ? sn : cs;
    if (iq & 2) s = -s;
    if ((iq + 1) & 2) c = -c;
    *sp = __double2float_rn(s);
    *cp = __double2float_rn(c);
}

__device__ __forceinline__ float cl_sinf(float x) { float s, c; cl_sincosf(x, &s, &c); return s; }
__device__ __forceinline__ float cl_cosf(float x) { float s, c; cl_sincosf(x, &s, &c); return c; }

// ---------------------------------------------------------------------------
// Transport parameters (flattened OpticalParams / Readout / TimeBinning / Box).
// ---------------------------------------------------------------------------
struct Physics {
    float L0, L1, L2;
    float n_crystal, n_coupling, abs_len, ray_len, wrap_R, sigma_alpha, pde;
    float inv_v;                 // n_crystal / c, ns per mm
    float cx, cy, r2, sur_R, pitch, bin_ns, tau;
    int32_t nx, ny, nbins, max_bounces;
    uint32_t key0, key1;
    uint8_t abs_finite, ray_finite, wrap_specular, air_gap;
    uint8_t disc, sur_specular, two_sided, pad_;
};

enum : int32_t { FACE_XP = 1, FACE_XM = 2, FACE_YP = 3, FACE_YM = 4, FACE_BACK = 5, FACE_FRONT = 6 };
enum : int32_t {
    ST_FLYING = 0, ST_DETECTED = 1, ST_ABS_BULK = 2, ST_ABS_WALL = 3,
    ST_ABS_SIPM = 4, ST_CAP = 5, ST_ABS_SUR = 6
};

constexpr float TWO_PI_F = 6.2831854820251465f;   // 2f0*Float32(pi), exact doubling
constexpr float C_MM_NS = 299.792458f;

// fresnel, src/optics.jl:10-19.  Returns tir; R set when !tir.
__device__ __forceinline__ bool fresnel(float n1, float n2, float cosi, float& R)
{
    const float q = n1 / n2;
    const float sin2t = (q * q) * (1.0f - cosi * cosi);
    if (sin2t >= 1.0f) { R = 1.0f; return true; }
    const float cost = sqrtf(1.0f - sin2t);
    const float a = (n1 * cosi - n2 * cost) / (n1 * cosi + n2 * cost);
    const float b = (n1 * cost - n2 * cosi) / (n1 * cost + n2 * cosi);
    R = 0.5f * (a * a + b * b);
    return false;
}

__device__ __forceinline__ int face_axis(int32_t face) { return face <= 2 ? 1 : (face <= 4 ? 2 : 3); }

__device__ __forceinline__ void specular(float& ux, float& uy, float& uz, int32_t face)
{
    const int a = face_axis(face);
    if (a == 1) ux = -ux; else if (a == 2) uy = -uy; else uz = -uz;
}

// lambertian_dir, src/optics.jl:118-138.
__device__ __forceinline__ void lambertian(Stream& s, const Physics& P, int32_t face,
                                           float& ux, float& uy, float& uz)
{
    const float ct = sqrtf(randu(s, P.key0, P.key1));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    const float phi = TWO_PI_F * randu(s, P.key0, P.key1);
    float sp, cp;
    cl_sincosf(phi, &sp, &cp);
    const float a = st * cp, b = st * sp;
    switch (face) {
    case FACE_XP:   ux = -ct; uy = a;   uz = b;   break;
    case FACE_XM:   ux = ct;  uy = a;   uz = b;   break;
    case FACE_YP:   ux = a;   uy = -ct; uz = b;   break;
    case FACE_YM:   ux = a;   uy = ct;  uz = b;   break;
    case FACE_BACK: ux = a;   uy = b;   uz = -ct; break;
    default:        ux = a;   uy = b;   uz = ct;  break;
    }
}

// gaussian, src/optics.jl:38-39.
__device__ __forceinline__ float gaussian(Stream& s, const Physics& P, const double2* tab)
{
    const float u1 = randu(s, P.key0, P.key1);
    const float l = cl_logf(u1, tab);
    const float u2 = randu(s, P.key0, P.key1);
    return sqrtf(-2.0f * l) * cl_cosf(TWO_PI_F * u2);
}

// surface_interact (UNIFIED specular lobe), src/optics.jl:49-81.
// Returns transmitted; on reflection the direction is updated.
__device__ __forceinline__ bool surface_interact(Stream& s, const Physics& P, const double2* tab,
                                                 float& ux, float& uy, float& uz, int32_t face)
{
    const int a = face_axis(face);
    const float sgn = (face == FACE_XP || face == FACE_YP || face == FACE_BACK) ? 1.0f : -1.0f;
    const float Nx = a == 1 ? sgn : 0.0f;
    const float Ny = a == 2 ? sgn : 0.0f;
    const float Nz = a == 3 ? sgn : 0.0f;
    for (int tries = 0; tries < 20; ++tries) {
        const float alpha = P.sigma_alpha * fabsf(gaussian(s, P, tab));
        if (alpha >= 1.2f) continue;
        float sa, ca;
        cl_sincosf(alpha, &sa, &ca);
        const float phi = TWO_PI_F * randu(s, P.key0, P.key1);
        float sp, cp;
        cl_sincosf(phi, &sp, &cp);
        const float b = sa * cp, c = sa * sp;
        const float Nfx = a == 1 ? ca * sgn : b;
        const float Nfy = a == 2 ? ca * sgn : (a == 1 ? b : c);
        const float Nfz = a == 3 ? ca * sgn : c;
        const float cosi = ux * Nfx + uy * Nfy + uz * Nfz;
        if (cosi <= 0.0f) continue;
        float R;
        const bool tir = fresnel(P.n_crystal, 1.0f, cosi, R);
        if (tir || randu(s, P.key0, P.key1) < R) {
            const float rx = ux - (2.0f * cosi) * Nfx;
            const float ry = uy - (2.0f * cosi) * Nfy;
            const float rz = uz - (2.0f * cosi) * Nfz;
            if (rx * Nx + ry * Ny + rz * Nz < 0.0f) {
                ux = rx; uy = ry; uz = rz;
                return false;
            }
        } else {
            return true;
        }
    }
    specular(ux, uy, uz, face);
    return false;
}

// rayleigh_dir, src/optics.jl:87-112.  The rejection loop accepts with
// probability >= 1/2 per pass; it is bounded for safety and reports a budget
// overrun through `overrun` (never reached with a proper uniform stream).
__device__ __forceinline__ void rayleigh(Stream& s, const Physics& P,
                                         float& ux, float& uy, float& uz, bool& overrun)
{
    float mu = 0.0f;
    int it = 0;
    for (;;) {
        mu = 1.0f - 2.0f * randu(s, P.key0, P.key1);
        if (2.0f * randu(s, P.key0, P.key1) <= 1.0f + mu * mu) break;
        if (++it >= 4096) { overrun = true; break; }
    }
    const float st = sqrtf(fmaxf(0.0f, 1.0f - mu * mu));
    const float phi = TWO_PI_F * randu(s, P.key0, P.key1);
    float sp, cp;
    cl_sincosf(phi, &sp, &cp);
    const float cb = st * cp, sb = st * sp;
    float t1x, t1y, t1z, inv;
    if (fabsf(uz) < 0.9f) {
        inv = 1.0f / sqrtf(ux * ux + uy * uy);
        t1x = -uy * inv; t1y = ux * inv; t1z = 0.0f;
    } else {
        inv = 1.0f / sqrtf(uy * uy + uz * uz);
        t1x = 0.0f; t1y = -uz * inv; t1z = uy * inv;
    }
    const float t2x = uy * t1z - uz * t1y;
    const float t2y = uz * t1x - ux * t1z;
    const float t2z = ux * t1y - uy * t1x;
    const float vx = mu * ux + cb * t1x + sb * t2x;
    const float vy = mu * uy + cb * t1y + sb * t2y;
    const float vz = mu * uz + cb * t1z + sb * t2z;
    inv = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
    ux = vx * inv; uy = vy * inv; uz = vz * inv;
}

// A photon in flight.
struct Photon {
    float x, y, z, ux, uy, uz, t;
    int32_t bounces, nscat;
    Stream rng;
};

// Photon generation (src/kernel.jl:162-180): isotropic direction
// (src/generation.jl:4-9), then t = pt + (-tau)*log(u) if tau > 0.
__device__ __forceinline__ void photon_start(Photon& ph, const Physics& P, const double2* tab,
                                             uint64_t pid, float x, float y, float z, float pt)
{
    stream_init(ph.rng, pid);
    ph.x = x; ph.y = y; ph.z = z;
    const float uz = 1.0f - 2.0f * randu(ph.rng, P.key0, P.key1);
    const float r = sqrtf(fmaxf(0.0f, 1.0f - uz * uz));
    const float phi = TWO_PI_F * randu(ph.rng, P.key0, P.key1);
    float sp, cp;
    cl_sincosf(phi, &sp, &cp);
    ph.ux = r * cp; ph.uy = r * sp; ph.uz = uz;
    float t = pt;
    if (P.tau > 0.0f) t += (-P.tau) * cl_logf(randu(ph.rng, P.key0, P.key1), tab);
    ph.t = t;
    ph.bounces = 0;
    ph.nscat = 0;
}

// One iteration of the bounce loop, src/transport.jl:126-233 /
// src/kernel.jl:185-299.  Returns the terminal status or ST_FLYING.  On
// detection `idx` receives the signed 1-based SiPM index.
__device__ __forceinline__ int32_t photon_step(Photon& ph, const Physics& P, const double2* tab,
                                               int32_t& idx, bool& overrun)
{
    float& x = ph.x; float& y = ph.y; float& z = ph.z;
    float& ux = ph.ux; float& uy = ph.uy; float& uz = ph.uz;
    Stream& s = ph.rng;

    // wall_hit, src/geometry.jl:19-32
    const float dx = ux > 0.0f ? (P.L0 - x) / ux : (ux < 0.0f ? (-x) / ux : __int_as_float(0x7f800000));
    const float dy = uy > 0.0f ? (P.L1 - y) / uy : (uy < 0.0f ? (-y) / uy : __int_as_float(0x7f800000));
    const float dz = uz > 0.0f ? (P.L2 - z) / uz : (uz < 0.0f ? (-z) / uz : __int_as_float(0x7f800000));
    float d;
    int32_t face;
    if (dx <= dy && dx <= dz) { d = dx; face = ux > 0.0f ? FACE_XP : FACE_XM; }
    else if (dy <= dz)        { d = dy; face = uy > 0.0f ? FACE_YP : FACE_YM; }
    else                      { d = dz; face = uz > 0.0f ? FACE_BACK : FACE_FRONT; }

    // bulk competition
    const float inf = __int_as_float(0x7f800000);
    float d_abs = inf, d_ray = inf;
    if (P.abs_finite) d_abs = (-P.abs_len) * cl_logf(randu(s, P.key0, P.key1), tab);
    if (P.ray_finite) d_ray = (-P.ray_len) * cl_logf(randu(s, P.key0, P.key1), tab);
    if (d_abs < d && d_abs <= d_ray) return ST_ABS_BULK;
    if (d_ray < d) {
        x += d_ray * ux; y += d_ray * uy; z += d_ray * uz;
        ph.t += d_ray * P.inv_v;
        rayleigh(s, P, ux, uy, uz, overrun);
        ph.nscat += 1;
        ph.bounces += 1;
        return ph.bounces >= P.max_bounces ? ST_CAP : ST_FLYING;
    }

    // advance to the wall: clamp, then snap the hit axis
    const float nx_ = x + d * ux, ny_ = y + d * uy, nz_ = z + d * uz;
    x = nx_ > P.L0 ? P.L0 : (nx_ < 0.0f ? 0.0f : nx_);
    y = ny_ > P.L1 ? P.L1 : (ny_ < 0.0f ? 0.0f : ny_);
    z = nz_ > P.L2 ? P.L2 : (nz_ < 0.0f ? 0.0f : nz_);
    const int a = face_axis(face);
    if (a == 1)      x = face == FACE_XP ? P.L0 : 0.0f;
    else if (a == 2) y = face == FACE_YP ? P.L1 : 0.0f;
    else             z = face == FACE_BACK ? P.L2 : 0.0f;
    ph.t += d * P.inv_v;
    const float cosi = a == 1 ? fabsf(ux) : (a == 2 ? fabsf(uy) : fabsf(uz));

    if (face == FACE_BACK || (P.two_sided && face == FACE_FRONT)) {
        // readout face, src/transport.jl:161-185
        float R;
        const bool tir = fresnel(P.n_crystal, P.n_coupling, cosi, R);
        if (tir || randu(s, P.key0, P.key1) < R) {
            specular(ux, uy, uz, face);
        } else if (!P.disc || (x - P.cx) * (x - P.cx) + (y - P.cy) * (y - P.cy) <= P.r2) {
            if (randu(s, P.key0, P.key1) <= P.pde) {
                int32_t ii = 1 + (int32_t)(x / P.pitch);
                int32_t jj = 1 + (int32_t)(y / P.pitch);
                ii = ii < P.nx ? ii : P.nx;
                jj = jj < P.ny ? jj : P.ny;
                const int32_t lin = (jj - 1) * P.nx + ii;
                idx = face == FACE_FRONT ? -lin : lin;
                return ST_DETECTED;
            }
            return ST_ABS_SIPM;
        } else if (randu(s, P.key0, P.key1) <= P.sur_R) {
            if (P.sur_specular) specular(ux, uy, uz, face);
            else lambertian(s, P, face, ux, uy, uz);
        } else {
            return ST_ABS_SUR;
        }
    } else if (!P.air_gap) {
        // front-painted wrap, src/transport.jl:186-198
        if (randu(s, P.key0, P.key1) <= P.wrap_R) {
            if (P.wrap_specular) specular(ux, uy, uz, face);
            else lambertian(s, P, face, ux, uy, uz);
        } else {
            return ST_ABS_WALL;
        }
    } else {
        // back-painted wrap, src/transport.jl:199-226
        bool transmitted = false;
        if (P.sigma_alpha > 0.0f) {
            transmitted = surface_interact(s, P, tab, ux, uy, uz, face);
        } else {
            float R;
            const bool tir = fresnel(P.n_crystal, 1.0f, cosi, R);
            if (tir || randu(s, P.key0, P.key1) < R) specular(ux, uy, uz, face);
            else transmitted = true;
        }
        if (transmitted) {
            if (randu(s, P.key0, P.key1) <= P.wrap_R) {
                if (P.wrap_specular) specular(ux, uy, uz, face);
                else lambertian(s, P, face, ux, uy, uz);
            } else {
                return ST_ABS_WALL;
            }
        }
    }
    ph.bounces += 1;
    return ph.bounces >= P.max_bounces ? ST_CAP : ST_FLYING;
}

// Order-preserving map of a float onto uint32 (for atomicMin on times).
__device__ __forceinline__ uint32_t float_key(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k)
{
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
constexpr uint32_t INF_KEY = 0xFF800000u;   // float_key(+Inf)

}  // namespace cl
