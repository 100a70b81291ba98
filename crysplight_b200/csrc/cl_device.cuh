// cl_device.cuh — device-side building blocks of the transport engine:
// Philox4x32-10 streams, Float32 elementary functions, and the per-photon
// physics primitives the transport kernel's state machine composes.
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

// The same rounds with the key schedule (k0 + r*W0, k1 + r*W1, r = 0..9)
// precomputed: rk[2r], rk[2r+1].  With rk in the constant bank the XORs take
// their key operand straight from it.
__device__ __forceinline__ uint4 philox4x32_10_rk(uint4 c, const uint32_t* __restrict__ rk)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)PHILOX_M0 * c.x;
        const uint64_t p1 = (uint64_t)PHILOX_M1 * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c = make_uint4(hi1 ^ c.y ^ rk[2 * r], lo1, hi0 ^ c.w ^ rk[2 * r + 1], lo0);
    }
    return c;
}

// randu, src/philox.jl:62: ((x >>> 8) + 1.0f0) * 2^-24, exact, in (0, 1].
// (x >> 8) < 2^24 converts exactly, and (f + 1) * 2^-24 = f * 2^-24 + 2^-24 is
// representable, so one fused multiply-add gives the same bits as the
// reference's add then multiply (neither rounds).
__device__ __forceinline__ float u32_to_randu(uint32_t x)
{
    return __fmaf_rn((float)(x >> 8), 0x1p-24f, 0x1p-24f);
}

// A photon's uniform stream (PhiloxStream, src/philox.jl:34-62): key = seed,
// counter = (pid lo, pid hi, block, 0).  The uniforms are buffered, already
// converted by randu, in a per-lane ring of RING_LEN floats in shared memory:
// word i of the lane at column `tid` sits at ring[(i % RING_LEN) * RING_STRIDE]
// (every access is bank-conflict free).  Blocks are generated ahead of use, at
// one convergent point of the warp loop; pop() consumes in order and peek(d)
// looks d words ahead, so the sequence of uniforms is exactly the reference's.
// 32 words (32 KB for 256 threads; rings of 28, 36, 40 and 48 words measured
// 3-15% slower on the BGO+ESR scan)
#ifndef CL_RING_LEN
#define CL_RING_LEN 32
#endif
constexpr int RING_LEN = CL_RING_LEN;
constexpr int RING_STRIDE = 256;      // columns: the largest block the kernels launch

struct Rng {
    uint32_t pid_lo, pid_hi, block;
    uint32_t head;   // index of the next unread word
    int cnt;         // buffered words
};

__device__ __forceinline__ void rng_init(Rng& r, uint64_t pid)
{
    r.pid_lo = (uint32_t)pid;
    r.pid_hi = (uint32_t)(pid >> 32);
    r.block = 0;
    r.head = 0;
    r.cnt = 0;
}

// Two consecutive blocks at once (independent Philox chains interleave).
// Requires cnt <= RING_LEN - 8.
__device__ __forceinline__ void rng_fill2(Rng& r, float* ring, const uint32_t* rk)
{
    const uint4 o = philox4x32_10_rk(make_uint4(r.pid_lo, r.pid_hi, r.block, 0u), rk);
    const uint4 q = philox4x32_10_rk(make_uint4(r.pid_lo, r.pid_hi, r.block + 1u, 0u), rk);
    r.block += 2u;
    const uint32_t w = r.head + (uint32_t)r.cnt;
    ring[((w + 0u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o.x);
    ring[((w + 1u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o.y);
    ring[((w + 2u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o.z);
    ring[((w + 3u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o.w);
    ring[((w + 4u) % RING_LEN) * RING_STRIDE] = u32_to_randu(q.x);
    ring[((w + 5u) % RING_LEN) * RING_STRIDE] = u32_to_randu(q.y);
    ring[((w + 6u) % RING_LEN) * RING_STRIDE] = u32_to_randu(q.z);
    ring[((w + 7u) % RING_LEN) * RING_STRIDE] = u32_to_randu(q.w);
    r.cnt += 8;
}

// NB consecutive blocks at once.  Requires cnt <= RING_LEN - 4 * NB.
template <int NB>
__device__ __forceinline__ void rng_fill(Rng& r, float* ring, const uint32_t* rk)
{
    uint4 o[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b)
        o[b] = philox4x32_10_rk(make_uint4(r.pid_lo, r.pid_hi, r.block + (uint32_t)b, 0u), rk);
    r.block += (uint32_t)NB;
    const uint32_t w = r.head + (uint32_t)r.cnt;
    if (RING_LEN % (4 * NB) == 0 && (RING_LEN & (RING_LEN - 1)) == 0) {
        // every fill writes 4*NB words and pops move head and cnt in step, so
        // the write position head + cnt stays a multiple of 4*NB: the block
        // never wraps and its stores sit at fixed offsets from its first word
        float* blk = ring + (size_t)(w & (uint32_t)(RING_LEN - 1)) * RING_STRIDE;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            blk[(4 * b + 0) * RING_STRIDE] = u32_to_randu(o[b].x);
            blk[(4 * b + 1) * RING_STRIDE] = u32_to_randu(o[b].y);
            blk[(4 * b + 2) * RING_STRIDE] = u32_to_randu(o[b].z);
            blk[(4 * b + 3) * RING_STRIDE] = u32_to_randu(o[b].w);
        }
        r.cnt += 4 * NB;
        return;
    }
#if CL_RING_WRAP
    // w < 2 RING_LEN: one conditional subtraction wraps each index
    auto at = [&](uint32_t k) -> float& {
        const uint32_t i = w + k;
        return ring[(i >= (uint32_t)RING_LEN ? i - (uint32_t)RING_LEN : i) * RING_STRIDE];
    };
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        at(4u * b + 0u) = u32_to_randu(o[b].x);
        at(4u * b + 1u) = u32_to_randu(o[b].y);
        at(4u * b + 2u) = u32_to_randu(o[b].z);
        at(4u * b + 3u) = u32_to_randu(o[b].w);
    }
#else
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        ring[((w + 4u * b + 0u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o[b].x);
        ring[((w + 4u * b + 1u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o[b].y);
        ring[((w + 4u * b + 2u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o[b].z);
        ring[((w + 4u * b + 3u) % RING_LEN) * RING_STRIDE] = u32_to_randu(o[b].w);
    }
#endif
    r.cnt += 4 * NB;
}

#ifndef CL_RING_WRAP
#define CL_RING_WRAP 1
#endif

__device__ __forceinline__ float rng_peek(const Rng& r, const float* ring, uint32_t d)
{
#if CL_RING_WRAP
    uint32_t i = r.head + d;                   // head < RING_LEN, d < RING_LEN
    i = i >= (uint32_t)RING_LEN ? i - (uint32_t)RING_LEN : i;
    return ring[i * RING_STRIDE];
#else
    return ring[((r.head + d) % RING_LEN) * RING_STRIDE];
#endif
}

// Pop the next uniform.  The warp loop keeps at least as many words buffered
// as one iteration can consume (checked once per iteration through cnt).
__device__ __forceinline__ float rng_pop(Rng& r, const float* ring)
{
#if CL_RING_WRAP
    const float u = ring[r.head * RING_STRIDE];
    r.head = r.head + 1u == (uint32_t)RING_LEN ? 0u : r.head + 1u;
#else
    const float u = ring[(r.head % RING_LEN) * RING_STRIDE];
    r.head += 1u;
#endif
    r.cnt -= 1;
    return u;
}

// A register-only stream for the diagnostics kernel (same sequence).
struct SimpleStream {
    uint32_t pid_lo, pid_hi, block, b0, b1, b2, b3;
    int n;
};

__device__ __forceinline__ float simple_randu(SimpleStream& s, uint32_t k0, uint32_t k1)
{
    if (s.n == 0) {
        const uint4 o = philox4x32_10(make_uint4(s.pid_lo, s.pid_hi, s.block, 0u), k0, k1);
        s.block += 1u;
        s.b0 = o.x; s.b1 = o.y; s.b2 = o.z; s.b3 = o.w;
        s.n = 4;
    }
    const uint32_t x = s.b0;
    s.b0 = s.b1; s.b1 = s.b2; s.b2 = s.b3;
    s.n -= 1;
    return u32_to_randu(x);
}

// ---------------------------------------------------------------------------
// Float32 elementary functions.  Each is evaluated in Float64 to about 2^-51
// relative error and rounded once, so it returns the correctly rounded
// Float32 except when the exact value lies within ~2^-51 of a rounding
// boundary.  Arguments outside the transport's domain take a slow path
// through the CUDA double-precision library functions.
// ---------------------------------------------------------------------------

// Out-of-domain arguments (never reached by the transport): CUDA's Float64
// functions, kept out of line so the hot loop stays small.
static __device__ __noinline__ float slow_logf(float x) { return __double2float_rn(log((double)x)); }
static __device__ __noinline__ float2 slow_sincosf(float x)
{
    const double xd = (double)x;
    return make_float2(__double2float_rn(sin(xd)), __double2float_rn(cos(xd)));
}

// Natural log.  Table-driven (Tang 1990): x = 2^e * m, m in [sqrt(1/2), sqrt(2)),
// m = F_j (1 + r) with F_j = 1 + j/64, ln x = e ln2 + ln F_j + log1p(r),
// |r| < 1/90, log1p by its Taylor series to r^8.
template <int STRIDE = 1>
__device__ __forceinline__ float cl_logf(float x, const double2* __restrict__ tab)
{
    const uint32_t b = __float_as_uint(x);
    if (b - 0x00800000u >= 0x7f000000u)       // not a positive normal finite float
        return slow_logf(x);
    int e = (int)(b >> 23) - 127;
    uint32_t mb = b & 0x007fffffu;
    const int hi = mb >= 0x3504f3u;          // m >= sqrt(2): use m/2, e+1
    e += hi;
    mb |= hi ? 0x3f000000u : 0x3f800000u;
    const double m = (double)__uint_as_float(mb);
    const int j = __double2int_rn((m - 1.0) * 64.0);
    const double F = 1.0 + (double)j * 0.015625;
    const double2 t = tab[(j - CLM_LOG_JMIN) * STRIDE];
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

// log of a uniform ((x>>8)+1)*2^-24: always a positive normal float, so the
// domain check of cl_logf is not needed.
template <int STRIDE = 1>
__device__ __forceinline__ float cl_logf_u(float x, const double2* __restrict__ tab)
{
    const uint32_t b = __float_as_uint(x);
    int e = (int)(b >> 23) - 127;
    uint32_t mb = b & 0x007fffffu;
    const int hi = mb >= 0x3504f3u;
    e += hi;
    mb |= hi ? 0x3f000000u : 0x3f800000u;
    const double m = (double)__uint_as_float(mb);
    const int j = __double2int_rn((m - 1.0) * 64.0);
    const double F = 1.0 + (double)j * 0.015625;
    const double2 t = tab[(j - CLM_LOG_JMIN) * STRIDE];
    const double r = (m - F) * t.x;
    double p = CLM_L8;
    p = fma(p, r, CLM_L7);
    p = fma(p, r, CLM_L6);
    p = fma(p, r, CLM_L5);
    p = fma(p, r, CLM_L4);
    p = fma(p, r, CLM_L3);
    p = fma(p, r, CLM_L2);
    const double lp = fma(p * r, r, r);
    const double res = fma((double)e, CLM_LN2, t.y) + lp;
    return __double2float_rn(res);
}

// sin and cos together, table-driven: x = j*delta + r with delta = 2 pi/256
// (two-term delta, |r| <= pi/256), (sin, cos)(j*delta) from a 256-entry table
// in shared memory, sin r and cos r - 1 by their Taylor series to r^7 and r^8,
// recombined as S + (S (cos r - 1) + C sin r) and C + (C (cos r - 1) - S sin r).
// The table-driven core for 0 <= x <= 1e4 (the transport passes azimuths
// 2*pi*u in (0, 2*pi] and facet tilts in [0, 1.2)); +0 maps to (+0, 1).
// The core's Float64 constants sit in the constant bank, so every Float64
// instruction takes its coefficient as an operand (a 64-bit immediate cannot
// be encoded and would first be moved into registers).
static __constant__ double c_sc_coef[10] = {CLM_SC_INV_DELTA, CLM_SC_DELTA_HI, CLM_SC_DELTA_LO, CLM_TS7,
                                            CLM_TS5, CLM_TS3, CLM_TC8, CLM_TC6, CLM_TC4, CLM_TC2};
#ifndef CL_SC_MAGIC_RINT
#define CL_SC_MAGIC_RINT 1
#endif

template <int STRIDE = 1>
__device__ __forceinline__ void cl_sincosf_core(float x, const double2* __restrict__ sctab,
                                                float* sp, float* cp)
{
    const double xd = (double)x;
#if CL_SC_MAGIC_RINT
    // rint by the 1.5*2^52 shift (round to nearest even, |q| < 2^51): the
    // integer sits in the low word of the shifted sum
    const double q = xd * c_sc_coef[0];
    const double sh = q + 0x1.8p52;
    const double n = sh - 0x1.8p52;
    const int ni = __double2loint(sh);
#else
    const double n = rint(xd * c_sc_coef[0]);
    const int ni = (int)n;
#endif
    double r = fma(-n, c_sc_coef[1], xd);
    r = fma(-n, c_sc_coef[2], r);
    const double2 sc = sctab[(ni & (CLM_SC_N - 1)) * STRIDE];
    const double r2 = r * r;
    double ps = fma(c_sc_coef[3], r2, c_sc_coef[4]);
    ps = fma(ps, r2, c_sc_coef[5]);
    const double sr = fma(r * r2, ps, r);
    double pc = fma(c_sc_coef[6], r2, c_sc_coef[7]);
    pc = fma(pc, r2, c_sc_coef[8]);
    pc = fma(pc, r2, c_sc_coef[9]);
    const double cm1 = r2 * pc;
    *sp = __double2float_rn(sc.x + fma(sc.x, cm1, sc.y * sr));
    *cp = __double2float_rn(sc.y + fma(sc.y, cm1, -(sc.x * sr)));
}

template <int STRIDE = 1>
__device__ __forceinline__ void cl_sincosf(float x, const double2* __restrict__ sctab,
                                           float* sp, float* cp)
{
    const double xd = (double)x;
    if (!(fabs(xd) <= 1.0e4)) {
        const float2 sc = slow_sincosf(x);
        *sp = sc.x;
        *cp = sc.y;
        return;
    }
    if (xd == 0.0) {                           // sin(+-0) = +-0, cos(+-0) = 1
        *sp = x;
        *cp = 1.0f;
        return;
    }
    const double n = rint(xd * CLM_SC_INV_DELTA);
    double r = fma(-n, CLM_SC_DELTA_HI, xd);
    r = fma(-n, CLM_SC_DELTA_LO, r);
    const double2 sc = sctab[((int)n & (CLM_SC_N - 1)) * STRIDE];
    const double r2 = r * r;
    double ps = fma(CLM_TS7, r2, CLM_TS5);
    ps = fma(ps, r2, CLM_TS3);
    const double sr = fma(r * r2, ps, r);      // sin r
    double pc = fma(CLM_TC8, r2, CLM_TC6);
    pc = fma(pc, r2, CLM_TC4);
    pc = fma(pc, r2, CLM_TC2);
    const double cm1 = r2 * pc;                // cos r - 1
    const double s = sc.x + fma(sc.x, cm1, sc.y * sr);
    const double c = sc.y + fma(sc.y, cm1, -(sc.x * sr));
    *sp = __double2float_rn(s);
    *cp = __double2float_rn(c);
}



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
    uint32_t rk[20];             // Philox round keys
    float qc2, qa2;              // (n_crystal/n_coupling)^2, (n_crystal/1)^2
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

// fresnel with (n1/n2)^2 precomputed (the same Float32 value the reference
// computes each call).
__device__ __forceinline__ bool fresnel_q2(float n1, float n2, float q2, float cosi, float& R)
{
    const float sin2t = q2 * (1.0f - cosi * cosi);
    if (sin2t >= 1.0f) { R = 1.0f; return true; }
    const float cost = sqrtf(1.0f - sin2t);
    const float a = (n1 * cosi - n2 * cost) / (n1 * cosi + n2 * cost);
    const float b = (n1 * cost - n2 * cosi) / (n1 * cost + n2 * cosi);
    R = 0.5f * (a * a + b * b);
    return false;
}

__device__ __forceinline__ int face_axis(int32_t face) { return face <= 2 ? 1 : (face <= 4 ? 2 : 3); }

// specular, src/optics.jl:25-28.
__device__ __forceinline__ void specular(float& ux, float& uy, float& uz, int32_t face)
{
    const int a = face_axis(face);
    // selects, not branches: a warp whose lanes hit different axes runs one path
    ux = a == 1 ? -ux : ux;
    uy = a == 2 ? -uy : uy;
    uz = a == 3 ? -uz : uz;
}

// Distance along one axis to the face the direction points at:
// u > 0 ? (L - p) / u : (u < 0 ? -p / u : Inf).  The numerator is selected
// first, so a warp whose lanes point both ways runs one division, not two.
__device__ __forceinline__ float axis_distance(float L, float p, float u)
{
    const float q = (u > 0.0f ? L - p : -p) / u;
    return (u > 0.0f || u < 0.0f) ? q : __int_as_float(0x7f800000);
}

// wall_hit, src/geometry.jl:19-32.
__device__ __forceinline__ int32_t wall_hit(const Physics& P, float x, float y, float z,
                                            float ux, float uy, float uz, float& d)
{
    const float dx = axis_distance(P.L0, x, ux);
    const float dy = axis_distance(P.L1, y, uy);
    const float dz = axis_distance(P.L2, z, uz);
    if (dx <= dy && dx <= dz) { d = dx; return ux > 0.0f ? FACE_XP : FACE_XM; }
    if (dy <= dz)             { d = dy; return uy > 0.0f ? FACE_YP : FACE_YM; }
    d = dz;
    return uz > 0.0f ? FACE_BACK : FACE_FRONT;
}

// Direction about the inward normal of a face from cos(theta) = ct and the
// azimuth's (sin, cos): the tail of lambertian_dir, src/optics.jl:119-137.
__device__ __forceinline__ void lambertian_from(int32_t face, float ct, float sphi, float cphi,
                                                float& ux, float& uy, float& uz)
{
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    const float a = st * cphi, b = st * sphi;
    // the inward normal component on the face's axis, (a, b) on the other two
    // in axis order (XP: (-ct, a, b), YM: (a, ct, b), BACK: (a, b, -ct), ...),
    // by selects
    const int ax = face_axis(face);
    const float n = (face == FACE_XP || face == FACE_YP || face == FACE_BACK) ? -ct : ct;
    ux = ax == 1 ? n : a;
    uy = ax == 1 ? a : (ax == 2 ? n : b);
    uz = ax == 3 ? n : b;
}

// The tail of rayleigh_dir, src/optics.jl:93-111: rotate u by the polar
// cosine mu about itself with the azimuth's (sin, cos).
__device__ __forceinline__ void rayleigh_rotate(float mu, float sphi, float cphi,
                                                float& ux, float& uy, float& uz)
{
    const float st = sqrtf(fmaxf(0.0f, 1.0f - mu * mu));
    const float cb = st * cphi, sb = st * sphi;
    // t1 = (-uy, ux, 0)/|(ux, uy)| if |uz| < 0.9, else (0, -uz, uy)/|(uy, uz)|:
    // the same operations on selected operands (one square root and division
    // for a warp whose lanes take both cases)
    const bool zlow = fabsf(uz) < 0.9f;
    const float pa = zlow ? ux : uy, pb = zlow ? uy : uz;
    float inv = 1.0f / sqrtf(pa * pa + pb * pb);
    const float t1x = zlow ? -pb * inv : 0.0f;
    const float t1y = zlow ? pa * inv : -pb * inv;
    const float t1z = zlow ? 0.0f : pa * inv;
    const float t2x = uy * t1z - uz * t1y;
    const float t2y = uz * t1x - ux * t1z;
    const float t2z = ux * t1y - uy * t1x;
    const float vx = mu * ux + cb * t1x + sb * t2x;
    const float vy = mu * uy + cb * t1y + sb * t2y;
    const float vz = mu * uz + cb * t1z + sb * t2z;
    inv = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
    ux = vx * inv; uy = vy * inv; uz = vz * inv;
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
