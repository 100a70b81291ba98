// cl_transport.cu — sm_100a transport kernels and the C-ABI of
// include/crysplight_cuda.h.
//
// Kernel design (B200):
//   * persistent grid: (#SM x resident CTAs) CTAs of 256 threads; every warp
//     claims photon chunks from a device work queue (one 64-bit atomic per
//     chunk) and each lane refills itself with the next photon the moment
//     its photon terminates, so long-bouncing photons never idle a warp;
//   * parameters travel as a __grid_constant__ kernel argument (constant
//     bank), the log table sits in shared memory;
//   * point mode: the nx*ny*(nbins+1) count tile and the nx*ny first-time
//     tile live in shared memory; detections are warp-aggregated with
//     __match_any_sync (one shared atomic per distinct bin per warp step),
//     first times use atomicMin on order-preserving uint32 keys; each CTA
//     flushes its tile once with coalesced global atomics and the last CTA
//     decodes the first-time keys in place;
//   * segment mode (scan points, 511 keV events): per-segment 8x8 maps and
//     first-time keys are reduced with warp-aggregated global atomics;
//     a finalize kernel decodes keys and sums npe.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <mutex>
#include <new>

#include <cuda_runtime.h>
#include <curand_philox4x32_x.h>

#include "../../include/crysplight_cuda.h"
#include "cl_device.cuh"
#include "cl_surrogate.cuh"

#define CL_VERSION_STRING "crysplight_b200 0.1.0 (sm_100a)"

namespace cl {

constexpr unsigned FULL = 0xffffffffu;
// The tables are replicated: entry e of copy c sits at [e * COPIES + c] and a
// lane reads copy (lane % COPIES), so the 16-byte reads of the 8 lanes that
// share a shared-memory wavefront hit distinct banks when COPIES = 8.
#ifndef CL_LOG_COPIES
#define CL_LOG_COPIES 1
#endif
#ifndef CL_SC_COPIES
#define CL_SC_COPIES 1
#endif
constexpr int LOG_COPIES = CL_LOG_COPIES;
constexpr int SC_COPIES = CL_SC_COPIES;
constexpr int SCTAB_BYTES = CLM_SC_N * 16 * SC_COPIES;
constexpr int LOGTAB_BYTES = ((CLM_LOG_NTAB * 16 * LOG_COPIES + 127) / 128) * 128 + SCTAB_BYTES;  // both tables

__constant__ double c_logtab[2 * CLM_LOG_NTAB] = { CLM_LOG_TAB_INIT };
__constant__ double c_sctab[2 * CLM_SC_N] = { CLM_SC_TAB_INIT };

// Copy the log and sincos tables into shared memory (the first LOGTAB_BYTES).
__device__ __forceinline__ void load_tables(unsigned char* smem, double2*& tab, double2*& sctab)
{
    sctab = reinterpret_cast<double2*>(smem);
    tab = reinterpret_cast<double2*>(smem + SCTAB_BYTES);
    for (int i = threadIdx.x; i < CLM_SC_N * SC_COPIES; i += blockDim.x) {
        const int e = i / SC_COPIES;
        sctab[i] = make_double2(c_sctab[2 * e], c_sctab[2 * e + 1]);
    }
    for (int i = threadIdx.x; i < CLM_LOG_NTAB * LOG_COPIES; i += blockDim.x) {
        const int e = i / LOG_COPIES;
        tab[i] = make_double2(c_logtab[2 * e], c_logtab[2 * e + 1]);
    }
}

struct KArgs {
    Physics P;
    uint64_t pid0;
    int64_t n;
    int32_t npos;
    int32_t warp_chunk;
    int32_t cells;        // nx*ny
    int32_t bins_total;   // nbins+1
    const float* px; const float* py; const float* pz; const float* pt;
    const int64_t* src_off; const int32_t* src_seg; int64_t n_src; int64_t n_seg;
    uint32_t* counts;     // point: cells*bins_total
    uint32_t* keys;       // point: cells; segments: cells*n_seg
    uint32_t* maps;       // segments: cells*n_seg
    unsigned long long* tsum;   // segments with moments (MODE 2): cells*n_seg
    unsigned long long* tsum2;
    unsigned long long* counters;  // 9 x int64, cl_counters order
    uint8_t* r_status; int16_t* r_idx; float* r_t; int32_t* r_bounces;
    unsigned long long* queue;
    unsigned long long* steps;
    unsigned int* done;
    unsigned int* err;
    const float* logtab;  // log of every uniform (k+1)*2^-24 at [k], or NULL: compute
    unsigned long long budget_ns;   // device time budget of the launch, 0 = none
};

// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int time_bin0(float t, const Physics& P)
{
    // 1 + unsafe_trunc(t / bin_ns), overflow -> nbins+1 (src/transport.jl:100-101), 0-based
    const float q = t / P.bin_ns;
    if (!(q < (float)P.nbins)) return P.nbins;
    const int b = (int)q;
    return b < 0 ? 0 : b;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Galloping search: largest s >= hint with off[s] <= k (off[n_src] = total).
__device__ __forceinline__ int64_t find_source(const int64_t* __restrict__ off, int64_t n_src,
                                               int64_t hint, int64_t k)
{
    int64_t lo = hint, step = 1;
    int64_t hi = hint + 1;
    while (hi < n_src && __ldg(off + hi) <= k) {
        lo = hi;
        step <<= 1;
        hi = lo + step;
    }
    if (hi > n_src) hi = n_src;
    // invariant: off[lo] <= k < off[hi]  (off[n_src] > k)
    while (hi - lo > 1) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(off + mid) <= k) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-lane transport states of the warp loop.  One loop iteration moves each
// active lane one state forward; a whole wall interaction (move, UNIFIED try,
// wrap) completes in one iteration, so an iteration is about one photon-step.
enum : int32_t {
    S_IDLE = 0,   // no photon
    S_INIT = 1,   // emission: direction and time (src/kernel.jl:173-180)
    S_MOVE = 2,   // bulk competition + wall interaction (src/transport.jl:127-233)
    S_UNI = 3,    // another UNIFIED try at the same wall (src/optics.jl:54-78)
    S_RAY = 4,    // Rayleigh rejection sampling + rotation (src/optics.jl:87-112)
    S_LAMB = 5,   // Lambertian re-injection (src/optics.jl:118-138)
};
// Uniforms one iteration can consume at most (move: abs, ray, 3 for the
// UNIFIED try, Fresnel, wrap; a Rayleigh frame: two tries of 2 and the
// azimuth).  The ring is topped up to this before the iteration's draws.
constexpr int DRAWS_PER_ITER = 7;
// Fresnel interfaces met in an iteration (one evaluation serves all three).
enum : int32_t { FK_NONE = 0, FK_READOUT = 1, FK_POLISHED = 2, FK_FACET = 3 };

#ifndef CL_FILL_JOIN
#define CL_FILL_JOIN 1
#endif
#ifndef CL_FILL_BLOCKS
#define CL_FILL_BLOCKS 2
#endif
#ifndef CL_USE_LOGTAB
#define CL_USE_LOGTAB 1
#endif
#ifndef CL_DEFAULT_WARP_CHUNK
#define CL_DEFAULT_WARP_CHUNK 0
#endif
#ifndef CL_CHUNKS_PER_WARP
#define CL_CHUNKS_PER_WARP 16
#endif
#ifndef CL_MAX_WARP_CHUNK
#define CL_MAX_WARP_CHUNK 256
#endif
#ifndef CL_MIN_CTAS_PER_SM
#define CL_MIN_CTAS_PER_SM 4
#endif

// Optical configurations compiled with their flags as constants (the branches
// they rule out vanish from the loop): SPEC_ESR and SPEC_TEFLON are a rough
// (UNIFIED) back-painted wrap, specular or Lambertian, over a full, one-sided
// readout face with finite absorption and Rayleigh lengths -- the BGO+ESR and
// CsI(Tl)+Teflon run files; SPEC_ANY reads every flag from the parameters.
enum : int { SPEC_ANY = 0, SPEC_ESR = 1, SPEC_TEFLON = 2 };

template <int MODE, bool REC, bool TILE, int SPEC>
__global__ void __launch_bounds__(256, CL_MIN_CTAS_PER_SM) transport_kernel(const __grid_constant__ KArgs A)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *s_tab, *s_sctab;
    load_tables(smem, s_tab, s_sctab);
    float* s_ring = reinterpret_cast<float*>(smem + LOGTAB_BYTES);
    uint32_t* s_counts = reinterpret_cast<uint32_t*>(s_ring + RING_LEN * RING_STRIDE);
    uint32_t* s_keys = s_counts + (TILE ? A.cells * A.bins_total : 0);
    __shared__ unsigned long long s_cnt[10];
    __shared__ unsigned int s_last;

    const Physics& P = A.P;
    const int tid = threadIdx.x;
    if (TILE) {
        const int nt = A.cells * A.bins_total;
        for (int i = tid; i < nt; i += blockDim.x) s_counts[i] = 0u;
        for (int i = tid; i < A.cells; i += blockDim.x) s_keys[i] = INF_KEY;
    }
    if (tid < 10) s_cnt[tid] = 0ull;
    __syncthreads();

    uint32_t* tile_counts = TILE ? s_counts : A.counts;
    uint32_t* tile_keys = TILE ? s_keys : A.keys;
    float* ring = s_ring + tid;

    const int lane = tid & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const double2* my_tab = s_tab + (lane % LOG_COPIES);
    const double2* my_sctab = s_sctab + (lane % SC_COPIES);
    const bool air_gap = SPEC != SPEC_ANY || P.air_gap;
    const bool uni_possible = SPEC != SPEC_ANY || (P.air_gap && P.sigma_alpha > 0.0f);
    const bool wrap_specular = SPEC == SPEC_ESR || (SPEC == SPEC_ANY && P.wrap_specular);
    const bool abs_finite = SPEC != SPEC_ANY || P.abs_finite;
    const bool ray_finite = SPEC != SPEC_ANY || P.ray_finite;
    const bool disc = SPEC == SPEC_ANY && P.disc;
    const bool two_sided = SPEC == SPEC_ANY && P.two_sided;
    // states and interfaces a configuration never reaches (tests on them compile away)
    constexpr bool lamb_possible = SPEC != SPEC_ESR;      // Lambertian wrap or surround
    constexpr bool polished_possible = SPEC == SPEC_ANY;  // back-painted face without roughness
    const float inf = __int_as_float(0x7f800000);

    // per-lane photon state
    float x = 0.f, y = 0.f, z = 0.f, ux = 0.f, uy = 0.f, uz = 0.f, t = 0.f;
    float carry = 0.f;                 // uz (init), mu (Rayleigh), u1 (Lambertian)
    int32_t bounces = 0, nscat = 0, st = S_IDLE, face = 0, tries = 0;
    Rng rng;
    rng_init(rng, 0);
    int64_t k = 0;
    int32_t seg = 0;
    // warp-uniform work pool
    int64_t pool_lo = 0, pool_hi = 0, pool_src = 0;
    bool exhausted = false;
    bool overrun = false, under = false, timed_out = false;
    // time budget: a warp-uniform iteration count, the clock read every 256
    uint32_t iter = 0;
    const unsigned long long t_begin = A.budget_ns ? globaltimer_ns() : 0ull;

    for (;;) {
        // ---- refill idle lanes from the warp's pool / the global queue ----
        const unsigned need = __ballot_sync(FULL, st == S_IDLE);
        if (need != 0u && !exhausted) {
            const int nneed = __popc(need);
            const int rank = __popc(need & lt_mask);
            int64_t my_k = -1;
            int64_t my_hint = pool_src;
            const int64_t avail = pool_hi - pool_lo;
            const int64_t taken = avail < nneed ? avail : (int64_t)nneed;
            if (st == S_IDLE && rank < taken) my_k = pool_lo + rank;
            pool_lo += taken;
            if (taken < nneed) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(A.queue, (unsigned long long)A.warp_chunk);
                base = __shfl_sync(FULL, base, 0);
                if ((int64_t)base >= A.n) {
                    exhausted = true;
                } else {
                    pool_lo = (int64_t)base;
                    pool_hi = pool_lo + A.warp_chunk;
                    if (pool_hi > A.n) pool_hi = A.n;
                    if (MODE != 0) {
                        int64_t s0 = 0;
                        if (lane == 0) s0 = find_source(A.src_off, A.n_src, pool_src, pool_lo);
                        pool_src = __shfl_sync(FULL, s0, 0);
                    }
                    const int64_t rem = nneed - taken;
                    const int64_t avail2 = pool_hi - pool_lo;
                    const int64_t taken2 = avail2 < rem ? avail2 : rem;
                    if (st == S_IDLE && rank >= taken && rank - taken < taken2) {
                        my_k = pool_lo + (rank - taken);
                        my_hint = pool_src;
                    }
                    pool_lo += taken2;
                }
            }
            if (my_k >= 0) {
                k = my_k;
                if (MODE == 0) {
                    const int32_t j = A.npos == 1 ? 0 : (int32_t)((uint64_t)k % (uint64_t)A.npos);
                    x = __ldg(A.px + j); y = __ldg(A.py + j); z = __ldg(A.pz + j);
                    t = A.pt ? __ldg(A.pt + j) : 0.0f;
                } else {
                    const int64_t s = find_source(A.src_off, A.n_src, my_hint, k);
                    x = __ldg(A.px + s); y = __ldg(A.py + s); z = __ldg(A.pz + s);
                    t = A.pt ? __ldg(A.pt + s) : 0.0f;
                    seg = __ldg(A.src_seg + s);
                }
                rng_init(rng, A.pid0 + (uint64_t)k + 1ull);
                bounces = 0; nscat = 0; tries = 0;
                st = S_INIT;
            }
        }
        if (!__any_sync(FULL, st != S_IDLE)) break;
        if (A.budget_ns != 0ull && ((++iter) & 255u) == 0u) {
            // photons still in flight are dropped; the host reports CL_ERR_TIMEOUT
            if (__any_sync(FULL, globaltimer_ns() - t_begin > A.budget_ns)) { timed_out = true; break; }
        }

        // ---- top up the uniform ring: one Philox call site for the warp ----
        {
            const bool want = st != S_IDLE && rng.cnt < DRAWS_PER_ITER;
            if (__any_sync(FULL, want)) {
#if CL_FILL_JOIN
                // every lane with room tops up at this convergent point, so
                // later iterations need the fill less often
                if (st != S_IDLE && rng.cnt <= RING_LEN - 4 * CL_FILL_BLOCKS)
                    rng_fill<CL_FILL_BLOCKS>(rng, ring, P.rk);
#else
                if (want) rng_fill2(rng, ring, P.rk);
#endif
            }
        }

        // ---- pre: draw uniforms, stage arguments of the elementary functions ----
        float a0 = 1.f, a1 = 1.f, a2 = 1.f, p0 = 1.f, p1 = 1.f;
        bool nl0 = false, nl1 = false, nl2 = false, ns0 = false, ns1 = false;
        bool ray_ok = false;
        if (st == S_INIT) {
            carry = 1.0f - 2.0f * rng_pop(rng, ring);       // uz
            p1 = TWO_PI_F * rng_pop(rng, ring); ns1 = true;  // azimuth
            if (P.tau > 0.0f) { a0 = rng_pop(rng, ring); nl0 = true; }
        } else if (st == S_MOVE || st == S_UNI) {
            if (st == S_MOVE) {
                if (abs_finite) { a0 = rng_pop(rng, ring); nl0 = true; }
                if (ray_finite) { a1 = rng_pop(rng, ring); nl1 = true; }
            }
            if (uni_possible) {
                // speculative: the next three uniforms are the UNIFIED try's
                // gaussian pair and facet azimuth if this step reaches a wrap
                a2 = rng_peek(rng, ring, 0u); nl2 = true;
                p0 = TWO_PI_F * rng_peek(rng, ring, 1u); ns0 = true;
                p1 = TWO_PI_F * rng_peek(rng, ring, 2u); ns1 = true;
            }
        } else if (st == S_RAY) {
            float mu = 1.0f - 2.0f * rng_pop(rng, ring);
            ray_ok = 2.0f * rng_pop(rng, ring) <= 1.0f + mu * mu;
            if (!ray_ok) {
                // a second try in the same iteration (the reference's next
                // draws, in order): 8 of 9 scatters end in one iteration
                ++tries;
                mu = 1.0f - 2.0f * rng_pop(rng, ring);
                ray_ok = 2.0f * rng_pop(rng, ring) <= 1.0f + mu * mu;
            }
            carry = mu;
            if (ray_ok) { p1 = TWO_PI_F * rng_pop(rng, ring); ns1 = true; }
        } else if (lamb_possible && st == S_LAMB) {
            carry = rng_pop(rng, ring);                       // u for cos(theta)
            p1 = TWO_PI_F * rng_pop(rng, ring); ns1 = true;
        }

        // ---- elementary functions, once per warp (Float64, rounded once) ----
        // Straight-line and unconditional: the five evaluations are independent,
        // so their Float64 dependency chains interleave (lanes that need none of
        // them get the harmless argument 1).
        float L0, L1, L2, s0, c0, s1, c1;
        if (A.logtab) {
            // the logs' arguments are uniforms (k+1)*2^-24: look them up
            // (issued before the sincos work so the loads overlap it)
            // (the index is clamped into the table whatever the argument)
            L0 = __ldg(A.logtab + min((uint32_t)(a0 * 16777216.0f) - 1u, 0xFFFFFFu));
            L1 = __ldg(A.logtab + min((uint32_t)(a1 * 16777216.0f) - 1u, 0xFFFFFFu));
            L2 = __ldg(A.logtab + min((uint32_t)(a2 * 16777216.0f) - 1u, 0xFFFFFFu));
        } else {
            L0 = cl_logf_u<LOG_COPIES>(a0, my_tab);
            L1 = cl_logf_u<LOG_COPIES>(a1, my_tab);
            L2 = cl_logf_u<LOG_COPIES>(a2, my_tab);
        }
        cl_sincosf_core<SC_COPIES>(p0, my_sctab, &s0, &c0);
        cl_sincosf_core<SC_COPIES>(p1, my_sctab, &s1, &c1);
        (void)nl0; (void)nl1; (void)nl2; (void)ns0; (void)ns1;

        // ---- post, part 1 ----
        int32_t status = ST_FLYING, idx = 0;
        bool uni = false, wall_done = false, to_wrap = false;
        int32_t fk = FK_NONE;                  // which Fresnel interface this lane meets
        float fn2 = 1.0f, fq2 = 1.0f, fcos = 1.0f;
        if (st == S_INIT) {
            const float r = sqrtf(fmaxf(0.0f, 1.0f - carry * carry));
            ux = r * c1; uy = r * s1; uz = carry;
            if (P.tau > 0.0f) t += (-P.tau) * L0;
            st = S_MOVE;
        } else if (st == S_MOVE) {
            float d;
            const int32_t f = wall_hit(P, x, y, z, ux, uy, uz, d);
            const float d_abs = abs_finite ? (-P.abs_len) * L0 : inf;
            const float d_ray = ray_finite ? (-P.ray_len) * L1 : inf;
            if (d_abs < d && d_abs <= d_ray) {
                status = ST_ABS_BULK;
            } else if (d_ray < d) {
                x += d_ray * ux; y += d_ray * uy; z += d_ray * uz;
                t += d_ray * P.inv_v;
                st = S_RAY;
                tries = 0;
            } else {
                // advance to the wall: clamp, then snap the hit axis (src/transport.jl:146-157)
                const float nx_ = x + d * ux, ny_ = y + d * uy, nz_ = z + d * uz;
                x = nx_ > P.L0 ? P.L0 : (nx_ < 0.0f ? 0.0f : nx_);
                y = ny_ > P.L1 ? P.L1 : (ny_ < 0.0f ? 0.0f : ny_);
                z = nz_ > P.L2 ? P.L2 : (nz_ < 0.0f ? 0.0f : nz_);
                const int a = face_axis(f);
                if (a == 1)      x = f == FACE_XP ? P.L0 : 0.0f;
                else if (a == 2) y = f == FACE_YP ? P.L1 : 0.0f;
                else             z = f == FACE_BACK ? P.L2 : 0.0f;
                t += d * P.inv_v;
                const float cosi = a == 1 ? fabsf(ux) : (a == 2 ? fabsf(uy) : fabsf(uz));
                face = f;
                if (f == FACE_BACK || (two_sided && f == FACE_FRONT)) {
                    // readout face, src/transport.jl:161-185: Fresnel below
                    fk = FK_READOUT; fn2 = P.n_coupling; fq2 = P.qc2; fcos = cosi;
                } else if (!air_gap) {
                    // front-painted wrap, src/transport.jl:186-198
                    if (rng_pop(rng, ring) <= P.wrap_R) {
                        if (wrap_specular) { specular(ux, uy, uz, f); wall_done = true; }
                        else st = S_LAMB;
                    } else {
                        status = ST_ABS_WALL;
                    }
                } else if (uni_possible) {
                    tries = 0;
                    uni = true;                      // UNIFIED lobe, below
                } else {
                    // polished back-painted face, src/transport.jl:206-212: Fresnel below
                    fk = FK_POLISHED; fn2 = 1.0f; fq2 = P.qa2; fcos = cosi;
                }
            }
        } else if (st == S_UNI) {
            uni = true;
        } else if (st == S_RAY) {
            if (ray_ok || ++tries >= 4096) {
                overrun |= !ray_ok;
                rayleigh_rotate(carry, s1, c1, ux, uy, uz);
                nscat += 1;
                bounces += 1;
                if (bounces >= P.max_bounces) status = ST_CAP;
                else st = S_MOVE;
            }
        } else if (lamb_possible && st == S_LAMB) {
            lambertian_from(face, sqrtf(carry), s1, c1, ux, uy, uz);
            wall_done = true;
        }

        // UNIFIED try, first half (src/optics.jl:55-56): the gaussian tilt
        bool facet = false;
        float alpha = 0.f;
        if (uni) {
            rng_pop(rng, ring);       // gaussian u1 (its log is L2)
            rng_pop(rng, ring);       // gaussian u2 (its cos is c0)
            alpha = P.sigma_alpha * fabsf(sqrtf(-2.0f * L2) * c0);
            if (alpha >= 1.2f) {
                if (++tries >= 20) { specular(ux, uy, uz, face); wall_done = true; st = S_MOVE; }
                else st = S_UNI;
            } else {
                rng_pop(rng, ring);   // facet azimuth (its sincos is s1, c1)
                facet = true;
            }
        }

        // ---- facet tilt sin/cos, once per warp ----
        float sa = 0.f, ca = 1.f;
        if (__any_sync(FULL, facet)) {
            cl_sincosf_core<SC_COPIES>(facet ? alpha : 1.0f, my_sctab, &sa, &ca);
        }

        // UNIFIED try, second half (src/optics.jl:57-66): the facet normal
        float Nfx = 0.f, Nfy = 0.f, Nfz = 0.f;
        bool retry = false;
        if (facet) {
            const int a = face_axis(face);
            const float sgn = (face == FACE_XP || face == FACE_YP || face == FACE_BACK) ? 1.0f : -1.0f;
            const float b = sa * c1, c = sa * s1;
            Nfx = a == 1 ? ca * sgn : b;
            Nfy = a == 2 ? ca * sgn : (a == 1 ? b : c);
            Nfz = a == 3 ? ca * sgn : c;
            const float cosi = ux * Nfx + uy * Nfy + uz * Nfz;
            if (cosi <= 0.0f) retry = true;
            else { fk = FK_FACET; fn2 = 1.0f; fq2 = P.qa2; fcos = cosi; }
        }

        // ---- Fresnel (src/optics.jl:10-19), one evaluation per warp ----
        float R = 1.0f;
        bool tir = true;
        if (__any_sync(FULL, fk != FK_NONE)) {
            if (fk != FK_NONE) tir = fresnel_q2(P.n_crystal, fn2, fq2, fcos, R);
        }
        if (fk != FK_NONE) {
            const bool refl = tir || rng_pop(rng, ring) < R;
            if (fk == FK_READOUT) {
                if (refl) {
                    specular(ux, uy, uz, face);
                    wall_done = true;
                } else if (!disc || (x - P.cx) * (x - P.cx) + (y - P.cy) * (y - P.cy) <= P.r2) {
                    if (rng_pop(rng, ring) <= P.pde) {
                        int32_t ii = 1 + (int32_t)(x / P.pitch);
                        int32_t jj = 1 + (int32_t)(y / P.pitch);
                        ii = ii < P.nx ? ii : P.nx;
                        jj = jj < P.ny ? jj : P.ny;
                        const int32_t lin = (jj - 1) * P.nx + ii;
                        idx = face == FACE_FRONT ? -lin : lin;
                        status = ST_DETECTED;
                    } else {
                        status = ST_ABS_SIPM;
                    }
                } else if (rng_pop(rng, ring) <= P.sur_R) {
                    if (P.sur_specular) { specular(ux, uy, uz, face); wall_done = true; }
                    else st = S_LAMB;
                } else {
                    status = ST_ABS_SUR;
                }
            } else if (polished_possible && fk == FK_POLISHED) {
                if (refl) { specular(ux, uy, uz, face); wall_done = true; }
                else to_wrap = true;
            } else {
                // facet: reflect about the facet normal; keep it only if it
                // points back into the crystal (src/optics.jl:68-77)
                if (refl) {
                    const int a = face_axis(face);
                    const float sgn = (face == FACE_XP || face == FACE_YP || face == FACE_BACK) ? 1.0f : -1.0f;
                    const float Nx = a == 1 ? sgn : 0.0f;
                    const float Ny = a == 2 ? sgn : 0.0f;
                    const float Nz = a == 3 ? sgn : 0.0f;
                    const float rx = ux - (2.0f * fcos) * Nfx;
                    const float ry = uy - (2.0f * fcos) * Nfy;
                    const float rz = uz - (2.0f * fcos) * Nfz;
                    if (rx * Nx + ry * Ny + rz * Nz < 0.0f) {
                        ux = rx; uy = ry; uz = rz;
                        wall_done = true;
                        st = S_MOVE;
                    } else {
                        retry = true;
                    }
                } else {
                    to_wrap = true;
                    st = S_MOVE;
                }
            }
        }
        if (retry) {
            if (++tries >= 20) { specular(ux, uy, uz, face); wall_done = true; st = S_MOVE; }
            else st = S_UNI;
        }

        // transmitted into the air gap: the reflector (src/transport.jl:214-225)
        if (to_wrap) {
            if (rng_pop(rng, ring) <= P.wrap_R) {
                if (wrap_specular) { specular(ux, uy, uz, face); wall_done = true; }
                else st = S_LAMB;
            } else {
                status = ST_ABS_WALL;
            }
        }

        under |= rng.cnt < 0;

        // end of a wall interaction: count the bounce (src/transport.jl:228-232)
        if (wall_done && status == ST_FLYING) {
            bounces += 1;
            if (bounces >= P.max_bounces) status = ST_CAP;
            else st = S_MOVE;
        }

        // ---- detections: warp-aggregated atomics ----
        const bool det = status == ST_DETECTED;
        const unsigned dmask = __ballot_sync(FULL, det);
        if (det) {
            const int32_t lin = idx < 0 ? -idx : idx;
            const int32_t cell = lin - 1;
            const uint32_t key = float_key(t);
            if (MODE == 0) {
                const int32_t slot = cell + A.cells * time_bin0(t, P);
                const unsigned g = __match_any_sync(dmask, slot);
                // one atomic per distinct slot: the group's count and its earliest time
                const uint32_t kmin = __reduce_min_sync(g, key);
                if (lane == __ffs(g) - 1) {
                    atomicAdd(tile_counts + slot, (uint32_t)__popc(g));
                    atomicMin(tile_keys + cell, kmin);
                }
            } else {
                // a segment id outside the maps (untrusted device input) drops the detection
                const bool seg_ok = seg >= 0 && (int64_t)seg < A.n_seg;
                const unsigned okmask = __ballot_sync(dmask, seg_ok);
                if (seg_ok) {
                    const unsigned long long slot =
                        (unsigned long long)seg * (unsigned long long)A.cells + (unsigned long long)cell;
                    const unsigned g = __match_any_sync(okmask, slot);
                    const uint32_t kmin = __reduce_min_sync(g, key);
                    if (lane == __ffs(g) - 1) {
                        atomicAdd(A.maps + slot, (uint32_t)__popc(g));
                        atomicMin(A.keys + slot, kmin);
                    }
                    if (MODE == 2) {
                        // fixed-point time moments (exact integer sums, order-independent)
                        const float tc = fminf(fmaxf(t, 0.0f), CL_MOMENT_T_MAX_NS);
                        atomicAdd(A.tsum + slot, __float2ull_rn(tc * CL_MOMENT_T_SCALE));
                        atomicAdd(A.tsum2 + slot, __float2ull_rn((tc * tc) * CL_MOMENT_T2_SCALE));
                    }
                } else {
                    atomicOr(A.err, 16u);
                }
            }
        }

        // ---- terminal bookkeeping: warp-aggregated counters ----
        const bool term = status != ST_FLYING;
        const unsigned tmask = __ballot_sync(FULL, term);
        if (tmask != 0u) {
            if (term) {
                const unsigned g = __match_any_sync(tmask, status);
                // counters[] order: ndet, ndet_front, bulk, wall, sipm, cap, sur
                const int slot = status == ST_DETECTED ? 0 : (status == ST_ABS_SUR ? 6 : status);
                if (lane == __ffs(g) - 1) atomicAdd(&s_cnt[slot], (unsigned long long)__popc(g));
                if (REC) {
                    if (A.r_status) A.r_status[k] = (uint8_t)status;
                    if (A.r_idx) A.r_idx[k] = (int16_t)idx;
                    if (A.r_t) A.r_t[k] = t;
                    if (A.r_bounces) A.r_bounces[k] = bounces;
                }
            }
            const unsigned front = __ballot_sync(FULL, det && idx < 0);
            const uint32_t sb = __reduce_add_sync(FULL, det ? (uint32_t)bounces : 0u);
            const uint32_t sc = __reduce_add_sync(FULL, term ? (uint32_t)nscat : 0u);
            const uint32_t ss = __reduce_add_sync(FULL, term ? (uint32_t)(bounces + (status != ST_CAP)) : 0u);
            if (lane == 0) {
                if (front) atomicAdd(&s_cnt[1], (unsigned long long)__popc(front));
                if (sc) atomicAdd(&s_cnt[7], (unsigned long long)sc);
                if (sb) atomicAdd(&s_cnt[8], (unsigned long long)sb);
                atomicAdd(&s_cnt[9], (unsigned long long)ss);
            }
            if (term) st = S_IDLE;
        }
    }
    if (overrun) atomicOr(A.err, 1u);
    if (under) atomicOr(A.err, 2u);
    if (timed_out && lane == 0) atomicOr(A.err, 32u);
    __syncthreads();

    // ---- one coalesced flush per CTA ----
    if (TILE) {
        const int nt = A.cells * A.bins_total;
        for (int i = tid; i < nt; i += blockDim.x) {
            const uint32_t v = s_counts[i];
            if (v) atomicAdd(A.counts + i, v);
        }
        for (int i = tid; i < A.cells; i += blockDim.x) {
            const uint32_t kk = s_keys[i];
            if (kk != INF_KEY) atomicMin(A.keys + i, kk);
        }
    }
    if (tid < 9) {
        const unsigned long long v = s_cnt[tid];
        if (v) atomicAdd(A.counters + tid, v);
    } else if (tid == 9) {
        const unsigned long long v = s_cnt[9];
        if (v) atomicAdd(A.steps, v);
    }

    if (MODE == 0) {
        // last CTA decodes the first-time keys into Float32 in place
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = (atomicAdd(A.done, 1u) == gridDim.x - 1u) ? 1u : 0u;
        __syncthreads();
        if (s_last) {
            __threadfence();
            for (int i = tid; i < A.cells; i += blockDim.x) {
                const uint32_t kk = __ldcg(A.keys + i);
                A.keys[i] = __float_as_uint(key_float(kk));
            }
        }
    }
}

// Zero the outputs and the work queue before a launch.
__global__ void init_kernel(uint32_t* counts, int64_t n_counts, uint32_t* keys, int64_t n_keys,
                            unsigned long long* counters, unsigned long long* queue,
                            unsigned long long* steps, unsigned int* done, unsigned int* err)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = i0; i < n_counts; i += stride) counts[i] = 0u;
    for (int64_t i = i0; i < n_keys; i += stride) keys[i] = INF_KEY;
    if (i0 < 9) counters[i0] = 0ull;
    if (i0 == 0) { *queue = 0ull; *steps = 0ull; *done = 0u; *err = 0u; }
}

// The log table of the uniforms: t[k] = cl_logf_u((k+1) * 2^-24), the same
// function and rounding as the computed path, for k < 2^24.
__global__ void logtab_fill(float* t)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *s_tab, *s_sctab;
    load_tables(smem, s_tab, s_sctab);
    __syncthreads();
    const double2* my_tab = s_tab + (threadIdx.x % LOG_COPIES);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < (1u << 24); k += gridDim.x * blockDim.x)
        t[k] = cl_logf_u<LOG_COPIES>(u32_to_randu(k << 8), my_tab);
}

// Segment mode: decode tmin keys in place and sum npe per segment.
__global__ void finalize_segments(const uint32_t* maps, uint32_t* keys, int32_t* npe,
                                  int64_t n_seg, int32_t cells)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = n_seg * cells;
    for (int64_t i = i0; i < total; i += stride) keys[i] = __float_as_uint(key_float(keys[i]));
    for (int64_t s = i0; s < n_seg; s += stride) {
        uint32_t acc = 0;
        const uint32_t* m = maps + s * cells;
        for (int c = 0; c < cells; ++c) acc += m[c];
        npe[s] = (int32_t)acc;
    }
}

__global__ void decode_keys_kernel(uint32_t* keys, int64_t n)
{
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) keys[i] = __float_as_uint(key_float(keys[i]));
}

// ---- diagnostics ----
__global__ void debug_math_kernel(int fn, const float* in, float* out, int64_t n)
{
    __shared__ __align__(16) unsigned char tabs[LOGTAB_BYTES];
    double2 *s_tab, *s_sctab;
    load_tables(tabs, s_tab, s_sctab);
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float x = in[i];
        float r;
        if (fn == 0) {
            r = cl_logf<LOG_COPIES>(x, s_tab + (threadIdx.x % LOG_COPIES));
        } else {
            float sv, cv;
            cl_sincosf<SC_COPIES>(x, s_sctab + (threadIdx.x % SC_COPIES), &sv, &cv);
            r = fn == 1 ? sv : cv;
        }
        out[i] = r;
    }
}

__global__ void debug_philox_kernel(int use_curand, const uint32_t* ctr, uint32_t* out, int64_t n,
                                    uint32_t k0, uint32_t k1)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint4 c = make_uint4(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]);
        uint4 o;
        if (use_curand) o = curand_Philox4x32_10(c, make_uint2(k0, k1));
        else o = philox4x32_10(c, k0, k1);
        out[4 * i] = o.x; out[4 * i + 1] = o.y; out[4 * i + 2] = o.z; out[4 * i + 3] = o.w;
    }
}

__global__ void debug_randu_kernel(float* out, int64_t n, int32_t n_per, uint32_t k0, uint32_t k1)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        SimpleStream s;
        const uint64_t pid = (uint64_t)i + 1ull;
        s.pid_lo = (uint32_t)pid; s.pid_hi = (uint32_t)(pid >> 32); s.block = 0; s.n = 0;
        s.b0 = s.b1 = s.b2 = s.b3 = 0;
        for (int32_t j = 0; j < n_per; ++j) out[i * n_per + j] = simple_randu(s, k0, k1);
    }
}

}  // namespace cl

// ===========================================================================
// Host side
// ===========================================================================
using namespace cl;

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

struct cl_handle {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    DevBuf logtab;                 // 2^24 floats, or empty: the kernels compute the logs
    char err[512] = {0};
    DevBuf src, out, rec, scratch, dbg;
    int ctas_per_sm = 0;
    int threads = 256;
    int warp_chunk = CL_DEFAULT_WARP_CHUNK;   // 0: automatic per launch
    int64_t last_steps = 0;
    int max_smem_optin = 0;
    int max_smem_per_sm = 0;
    unsigned long long budget_ns = (unsigned long long)(CL_DEFAULT_TIME_BUDGET_S * 1e9);
};

static thread_local char g_create_err[512];

__attribute__((format(printf, 3, 4)))
static int set_err(cl_handle* h, int code, const char* fmt, ...)
{
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err, sizeof h->err, fmt, ap);
        va_end(ap);
    }
    return code;
}

static int cuda_fail(cl_handle* h, cudaError_t e, const char* what)
{
    cudaGetLastError();  // clear sticky non-fatal error
    return set_err(h, e == cudaErrorMemoryAllocation ? CL_ERR_OOM : CL_ERR_CUDA,
                   "%s: %s", what, cudaGetErrorString(e));
}

#define CK(h, call, what)                                   \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, (what)); \
    } while (0)

static int ensure(cl_handle* h, DevBuf& b, size_t bytes)
{
    if (bytes <= b.cap) return CL_OK;
    if (b.p) { cudaFree(b.p); b.p = nullptr; b.cap = 0; }
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(h, CL_ERR_OOM, "device allocation of %zu bytes failed", want);
    }
    b.cap = want;
    return CL_OK;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Allow dynamic shared memory up to the opt-in limit minus the kernel's
// static shared memory (their sum may not exceed the limit).
template <int MODE, bool REC, bool TILE, int SPEC>
static void set_kernel_attrs_spec(int smem_optin)
{
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, transport_kernel<MODE, REC, TILE, SPEC>) != cudaSuccess) return;
    cudaFuncSetAttribute(transport_kernel<MODE, REC, TILE, SPEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         smem_optin - (int)fa.sharedSizeBytes);
}

template <int MODE, bool REC, bool TILE>
static void set_kernel_attrs(int smem_optin)
{
    set_kernel_attrs_spec<MODE, REC, TILE, SPEC_ANY>(smem_optin);
    set_kernel_attrs_spec<MODE, REC, TILE, SPEC_ESR>(smem_optin);
    set_kernel_attrs_spec<MODE, REC, TILE, SPEC_TEFLON>(smem_optin);
}

extern "C" {

const char* cl_version(void) { return CL_VERSION_STRING; }
int cl_abi_version(void) { return CL_ABI_VERSION; }

int cl_create(cl_handle** out, int device)
{
    g_create_err[0] = 0;
    if (!out) {
        snprintf(g_create_err, sizeof g_create_err, "cl_create: null output pointer");
        return CL_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        snprintf(g_create_err, sizeof g_create_err, "cl_create: CUDA device %d unavailable (%s)",
                 device, e != cudaSuccess ? cudaGetErrorString(e) : "no such device");
        return e != cudaSuccess ? CL_ERR_CUDA : CL_ERR_ARG;
    }
    cl_handle* h = new (std::nothrow) cl_handle();
    if (!h) {
        snprintf(g_create_err, sizeof g_create_err, "cl_create: out of host memory");
        return CL_ERR_OOM;
    }
    h->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&h->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&h->max_smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaGetLastError();
        snprintf(g_create_err, sizeof g_create_err, "cl_create: %s", cudaGetErrorString(e));
        delete h;
        return CL_ERR_CUDA;
    }
    set_kernel_attrs<0, false, true>(h->max_smem_optin);
    set_kernel_attrs<0, true, true>(h->max_smem_optin);
    set_kernel_attrs<0, false, false>(h->max_smem_optin);
    set_kernel_attrs<0, true, false>(h->max_smem_optin);
    set_kernel_attrs<1, false, false>(h->max_smem_optin);
    set_kernel_attrs<1, true, false>(h->max_smem_optin);
    set_kernel_attrs<2, false, false>(h->max_smem_optin);
    cudaGetLastError();
    if (ensure(h, h->scratch, 64) != CL_OK) {
        snprintf(g_create_err, sizeof g_create_err, "cl_create: %s", h->err);
        cudaStreamDestroy(h->stream);
        delete h;
        return CL_ERR_OOM;
    }
#if CL_USE_LOGTAB
    // 64 MB table of the logs of all 2^24 uniforms; without it (allocation
    // failure) the kernels evaluate the same function in place
    if (cudaMalloc(&h->logtab.p, sizeof(float) << 24) == cudaSuccess) {
        h->logtab.cap = sizeof(float) << 24;
        logtab_fill<<<h->num_sms * 4, 256, LOGTAB_BYTES, h->stream>>>((float*)h->logtab.p);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(h->logtab.p);
            h->logtab = DevBuf();
        }
    } else {
        cudaGetLastError();
        h->logtab = DevBuf();
    }
#endif
    *out = h;
    return CL_OK;
}

void cl_destroy(cl_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    DevBuf* bufs[] = {&h->src, &h->out, &h->rec, &h->scratch, &h->dbg, &h->logtab};
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char* cl_last_error(const cl_handle* h) { return h ? h->err : g_create_err; }

int64_t cl_last_steps(const cl_handle* h) { return h ? h->last_steps : 0; }

int cl_set_launch(cl_handle* h, int ctas_per_sm, int threads_per_cta, int warp_chunk)
{
    if (!h) return CL_ERR_STATE;
    if (ctas_per_sm < 0 || ctas_per_sm > 32) return set_err(h, CL_ERR_ARG, "ctas_per_sm out of range");
    if (threads_per_cta != 0 && (threads_per_cta < 32 || threads_per_cta > 256 || threads_per_cta % 32))
        return set_err(h, CL_ERR_ARG, "threads_per_cta must be a multiple of 32 in [32, 256]");
    if (warp_chunk != 0 && (warp_chunk < 32 || warp_chunk > (1 << 20)))
        return set_err(h, CL_ERR_ARG, "warp_chunk must be in [32, 2^20]");
    h->ctas_per_sm = ctas_per_sm;
    h->threads = threads_per_cta ? threads_per_cta : 256;
    h->warp_chunk = warp_chunk ? warp_chunk : CL_DEFAULT_WARP_CHUNK;
    return CL_OK;
}

int cl_set_time_budget(cl_handle* h, double seconds)
{
    if (!h) return CL_ERR_STATE;
    if (!(seconds >= 0.0) || !std::isfinite(seconds) || seconds > 1.0e9)
        return set_err(h, CL_ERR_ARG, "time budget must be finite, >= 0 and <= 1e9 s");
    h->budget_ns = (unsigned long long)(seconds * 1e9);
    return CL_OK;
}

}  // extern "C"

// ---- argument validation shared by the entry points ----
static int check_params(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                        const cl_readout* ro, const cl_time_binning* tb, float tau_ns,
                        int32_t max_bounces)
{
    if (!box || !op || !ro || !tb) return set_err(h, CL_ERR_ARG, "null parameter struct");
    if (max_bounces > CL_MAX_BOUNCES_LIMIT)
        return set_err(h, CL_ERR_ARG, "max_bounces %d above the limit %d", (int)max_bounces,
                       (int)CL_MAX_BOUNCES_LIMIT);
    for (int i = 0; i < 3; ++i)
        if (!(box->L[i] > 0.0f) || !std::isfinite(box->L[i]))
            return set_err(h, CL_ERR_ARG, "box sizes must be finite and positive");
    if (ro->grid.nx < 1 || ro->grid.ny < 1 || (int64_t)ro->grid.nx * ro->grid.ny > 32767)
        return set_err(h, CL_ERR_ARG, "SiPM grid must have 1 <= nx*ny <= 32767");
    if (!(ro->grid.pitch_mm > 0.0f)) return set_err(h, CL_ERR_ARG, "pitch_mm must be positive");
    if (tb->nbins < 0 || tb->nbins > (1 << 24) || !(tb->bin_ns > 0.0f))
        return set_err(h, CL_ERR_ARG, "time binning needs bin_ns > 0 and 0 <= nbins <= 2^24");
    if (!(op->n_crystal > 0.0f) || !(op->n_coupling > 0.0f))
        return set_err(h, CL_ERR_ARG, "refractive indices must be positive");
    if (std::isnan(op->abs_len_mm) || std::isnan(op->rayleigh_mm) || std::isnan(op->wrap_R) ||
        std::isnan(op->sigma_alpha) || std::isnan(op->pde) || std::isnan(tau_ns) || std::isinf(tau_ns))
        return set_err(h, CL_ERR_ARG, "NaN/Inf in optical parameters or tau_ns");
    return CL_OK;
}

static Physics make_physics(const cl_box* box, const cl_optical_params* op, const cl_readout* ro,
                            const cl_time_binning* tb, float tau_ns, int32_t max_bounces, uint64_t seed)
{
    Physics P;
    memset(&P, 0, sizeof P);
    P.L0 = box->L[0]; P.L1 = box->L[1]; P.L2 = box->L[2];
    P.n_crystal = op->n_crystal; P.n_coupling = op->n_coupling;
    P.abs_len = op->abs_len_mm; P.ray_len = op->rayleigh_mm;
    P.wrap_R = op->wrap_R; P.sigma_alpha = op->sigma_alpha; P.pde = op->pde;
    P.inv_v = op->n_crystal / 299.792458f;
    P.cx = ro->cx; P.cy = ro->cy; P.r2 = ro->r2; P.sur_R = ro->sur_R;
    P.pitch = ro->grid.pitch_mm; P.bin_ns = tb->bin_ns; P.tau = tau_ns;
    P.nx = ro->grid.nx; P.ny = ro->grid.ny; P.nbins = tb->nbins; P.max_bounces = max_bounces;
    P.key0 = (uint32_t)seed; P.key1 = (uint32_t)(seed >> 32);
    {
        uint32_t k0 = P.key0, k1 = P.key1;
        for (int r = 0; r < 10; ++r) {
            P.rk[2 * r] = k0; P.rk[2 * r + 1] = k1;
            k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
        }
        const float qc = op->n_crystal / op->n_coupling;   // IEEE division on the host, as on the device
        const float qa = op->n_crystal / 1.0f;
        P.qc2 = qc * qc;
        P.qa2 = qa * qa;
    }
    P.abs_finite = std::isfinite(op->abs_len_mm) ? 1 : 0;
    P.ray_finite = std::isfinite(op->rayleigh_mm) ? 1 : 0;
    P.wrap_specular = op->wrap_specular ? 1 : 0;
    P.air_gap = op->air_gap ? 1 : 0;
    P.disc = ro->disc ? 1 : 0;
    P.sur_specular = ro->sur_specular ? 1 : 0;
    P.two_sided = ro->two_sided ? 1 : 0;
    return P;
}

// Scratch words: [0] queue u64, [1] steps u64, [2] done u32 | err u32
struct Scratch {
    unsigned long long* queue;
    unsigned long long* steps;
    unsigned int* done;
    unsigned int* err;
};

static Scratch scratch_of(cl_handle* h)
{
    unsigned long long* base = (unsigned long long*)h->scratch.p;
    Scratch s;
    s.queue = base;
    s.steps = base + 1;
    s.done = (unsigned int*)(base + 2);
    s.err = s.done + 1;
    return s;
}

// The compiled configuration a launch can use (SPEC_ANY where none matches).
static int spec_of(const Physics& P)
{
    if (!P.air_gap || !(P.sigma_alpha > 0.0f) || P.disc || P.two_sided || !P.abs_finite || !P.ray_finite)
        return SPEC_ANY;
    return P.wrap_specular ? SPEC_ESR : SPEC_TEFLON;
}

template <int MODE, bool REC, bool TILE, int SPEC>
static int launch_transport_spec(cl_handle* h, const KArgs& a, size_t smem, cudaStream_t st)
{
    auto kern = transport_kernel<MODE, REC, TILE, SPEC>;
    int per_sm = 0;
    CK(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, h->threads, smem), "occupancy");
    if (per_sm < 1) return set_err(h, CL_ERR_ARG, "transport kernel does not fit on an SM (shared tile too large)");
    if (h->ctas_per_sm > 0 && h->ctas_per_sm < per_sm) per_sm = h->ctas_per_sm;
    int64_t grid = (int64_t)h->num_sms * per_sm;
    KArgs b = a;
    if (b.warp_chunk <= 0) {
        // automatic: the largest chunk (fewest queue atomics) that still gives
        // every resident warp about CL_CHUNKS_PER_WARP chunks, so the end of
        // the queue stays balanced; between 32 and CL_MAX_WARP_CHUNK photons
        const int64_t warps = grid * (h->threads / 32);
        int64_t c = a.n / (warps * CL_CHUNKS_PER_WARP);
        c = c < 32 ? 32 : (c > CL_MAX_WARP_CHUNK ? CL_MAX_WARP_CHUNK : c);
        b.warp_chunk = (int32_t)(c & ~(int64_t)31);
    }
    // no more CTAs than warps' worth of first chunks
    const int64_t warps_needed = (b.n + b.warp_chunk - 1) / b.warp_chunk;
    const int64_t ctas_needed = (warps_needed + (h->threads / 32) - 1) / (h->threads / 32);
    if (grid > ctas_needed) grid = ctas_needed > 0 ? ctas_needed : 1;
    kern<<<(unsigned)grid, h->threads, smem, st>>>(b);
    CK(h, cudaGetLastError(), "transport kernel launch");
    return CL_OK;
}

template <int MODE, bool REC, bool TILE>
static int launch_transport(cl_handle* h, const KArgs& a, size_t smem, cudaStream_t st)
{
    switch (spec_of(a.P)) {
    case SPEC_ESR: return launch_transport_spec<MODE, REC, TILE, SPEC_ESR>(h, a, smem, st);
    case SPEC_TEFLON: return launch_transport_spec<MODE, REC, TILE, SPEC_TEFLON>(h, a, smem, st);
    default: return launch_transport_spec<MODE, REC, TILE, SPEC_ANY>(h, a, smem, st);
    }
}

static int enqueue_point(cl_handle* h, const Physics& P, const float* px, const float* py,
                         const float* pz, const float* pt, int32_t npos, int64_t n, uint64_t pid0,
                         uint32_t* counts, uint32_t* keys, unsigned long long* counters,
                         const cl_records* rec, cudaStream_t st)
{
    const int cells = P.nx * P.ny;
    const int bins_total = P.nbins + 1;
    const int64_t n_counts = (int64_t)cells * bins_total;
    Scratch s = scratch_of(h);
    init_kernel<<<(unsigned)std::min<int64_t>((n_counts + 255) / 256 + 1, 4096), 256, 0, st>>>(
        counts, n_counts, keys, cells, counters, s.queue, s.steps, s.done, s.err);
    CK(h, cudaGetLastError(), "init kernel launch");
    if (n == 0) {
        // no photons: decode the +Inf keys into Float32 +Inf
        decode_keys_kernel<<<1, 256, 0, st>>>(keys, cells);
        CK(h, cudaGetLastError(), "decode launch");
        return CL_OK;
    }
    KArgs a;
    memset(&a, 0, sizeof a);
    a.P = P; a.pid0 = pid0; a.n = n; a.npos = npos; a.warp_chunk = h->warp_chunk;
    a.cells = cells; a.bins_total = bins_total;
    a.px = px; a.py = py; a.pz = pz; a.pt = pt;
    a.counts = counts; a.keys = keys; a.counters = counters;
    const bool want_rec = rec && (rec->status || rec->idx || rec->t || rec->bounces);
    if (want_rec) { a.r_status = rec->status; a.r_idx = rec->idx; a.r_t = rec->t; a.r_bounces = rec->bounces; }
    a.queue = s.queue; a.steps = s.steps; a.done = s.done; a.err = s.err;
    a.logtab = (const float*)h->logtab.p;
    a.budget_ns = h->budget_ns;
    const size_t tile_bytes = ((size_t)n_counts + cells) * sizeof(uint32_t);
    const size_t base_bytes = LOGTAB_BYTES + (size_t)RING_LEN * RING_STRIDE * sizeof(float);
    // the shared-memory histogram tile only where it still leaves room for 4
    // CTAs per SM: with fewer resident warps the loop issues less often, which
    // costs more than the tile saves in global atomics (10^6-photon point
    // source, 8x8x81 bins: 879 M photons/s on global atomics at 4 CTAs/SM,
    // 843 M with the tile at 3)
    const size_t per_cta = base_bytes + tile_bytes + 1024;
    const bool tile = base_bytes + tile_bytes <= (size_t)std::min(h->max_smem_optin, 160 * 1024) &&
                      4 * per_cta <= (size_t)h->max_smem_per_sm;
    const size_t smem = base_bytes + (tile ? tile_bytes : 0);
    if (tile) return want_rec ? launch_transport<0, true, true>(h, a, smem, st)
                              : launch_transport<0, false, true>(h, a, smem, st);
    return want_rec ? launch_transport<0, true, false>(h, a, smem, st)
                    : launch_transport<0, false, false>(h, a, smem, st);
}

static int enqueue_segments(cl_handle* h, const Physics& P, const float* sx, const float* sy,
                            const float* sz, const float* sT, const int64_t* off, const int32_t* segid,
                            int64_t n_src, int64_t n_seg, int64_t n, uint64_t pid0,
                            uint32_t* maps, uint32_t* keys, int32_t* npe,
                            unsigned long long* counters, const cl_records* rec, cudaStream_t st,
                            unsigned long long* tsum = nullptr, unsigned long long* tsum2 = nullptr,
                            const SurSampleArgs* sample = nullptr)
{
    const int cells = P.nx * P.ny;
    const int64_t total = (int64_t)cells * n_seg;
    Scratch s = scratch_of(h);
    init_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256 + 1, 8192), 256, 0, st>>>(
        maps, total, keys, total, counters, s.queue, s.steps, s.done, s.err);
    CK(h, cudaGetLastError(), "init kernel launch");
    const bool moments = tsum && tsum2;
    if (moments) {
        CK(h, cudaMemsetAsync(tsum, 0, (size_t)total * sizeof(unsigned long long), st), "zero moments");
        CK(h, cudaMemsetAsync(tsum2, 0, (size_t)total * sizeof(unsigned long long), st), "zero moments");
    }
    if (n > 0) {
        KArgs a;
        memset(&a, 0, sizeof a);
        a.P = P; a.pid0 = pid0; a.n = n; a.npos = 1; a.warp_chunk = h->warp_chunk;
        a.cells = cells; a.bins_total = P.nbins + 1;
        a.px = sx; a.py = sy; a.pz = sz; a.pt = sT;
        a.src_off = off; a.src_seg = segid; a.n_src = n_src; a.n_seg = n_seg;
        a.keys = keys; a.maps = maps; a.counters = counters;
        const bool want_rec = rec && (rec->status || rec->idx || rec->t || rec->bounces);
        if (want_rec) { a.r_status = rec->status; a.r_idx = rec->idx; a.r_t = rec->t; a.r_bounces = rec->bounces; }
        a.queue = s.queue; a.steps = s.steps; a.done = s.done; a.err = s.err;
        a.logtab = (const float*)h->logtab.p;
        a.budget_ns = h->budget_ns;
        const size_t smem = LOGTAB_BYTES + (size_t)RING_LEN * RING_STRIDE * sizeof(float);
        a.tsum = tsum; a.tsum2 = tsum2;
        const int rc = moments ? launch_transport<2, false, false>(h, a, smem, st)
                     : want_rec ? launch_transport<1, true, false>(h, a, smem, st)
                                : launch_transport<1, false, false>(h, a, smem, st);
        if (rc != CL_OK) return rc;
    }
    if (sample) {
        SurSampleArgs sa = *sample;
        sa.maps = maps; sa.keys = keys; sa.err = s.err;
        CK(h, launch_surrogate_sample(sa, h->num_sms, st), "surrogate sampler launch");
    }
    finalize_segments<<<(unsigned)std::min<int64_t>((total + 255) / 256 + 1, 8192), 256, 0, st>>>(
        maps, keys, npe, n_seg, cells);
    CK(h, cudaGetLastError(), "finalize launch");
    return CL_OK;
}

static int collect(cl_handle* h, cudaStream_t st)
{
    Scratch s = scratch_of(h);
    unsigned long long steps = 0;
    unsigned int err = 0;
    CK(h, cudaMemcpyAsync(&steps, s.steps, sizeof steps, cudaMemcpyDeviceToHost, st), "copy steps");
    CK(h, cudaMemcpyAsync(&err, s.err, sizeof err, cudaMemcpyDeviceToHost, st), "copy status");
    CK(h, cudaStreamSynchronize(st), "stream synchronize");
    h->last_steps = (int64_t)steps;
    if (err & 32u)
        return set_err(h, CL_ERR_TIMEOUT, "the transport ran past the handle's time budget (%.3g s); "
                       "its outputs are incomplete", (double)h->budget_ns * 1e-9);
    if (err & 2u) return set_err(h, CL_ERR_CUDA, "internal error: uniform ring underflow in the transport kernel");
    if (err & 16u) return set_err(h, CL_ERR_ARG, "a source's segment id is out of range (its detections were dropped)");
    if (err & 8u) return set_err(h, CL_ERR_ARG, "a surrogate site's segment id is out of range (site skipped)");
    if (err & 4u) return set_err(h, CL_ERR_TIMEOUT, "a loop budget of the surrogate sampler ran out");
    if (err) return set_err(h, CL_ERR_TIMEOUT, "a device-side loop budget ran out (Rayleigh rejection sampler)");
    return CL_OK;
}

extern "C" {

int cl_run_photons(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                   const cl_readout* ro, const cl_time_binning* tb,
                   const float* px, const float* py, const float* pz,
                   const float* pt, int32_t npos,
                   int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                   float tau_ns, int32_t max_bounces,
                   uint32_t* counts, float* first_ns, cl_counters* counters,
                   const cl_records* records)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    if (npos < 1 || !px || !py || !pz) return set_err(h, CL_ERR_ARG, "need npos >= 1 source positions");
    if (n_photons < 0) return set_err(h, CL_ERR_ARG, "n_photons must be >= 0");
    if (!counts || !first_ns || !counters) return set_err(h, CL_ERR_ARG, "null output buffer");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = h->stream;

    const int cells = ro->grid.nx * ro->grid.ny;
    const size_t n_counts = (size_t)cells * (size_t)(tb->nbins + 1);
    // device layout: sources | counts | keys | counters ; records separately
    const size_t b_src = align256(4 * (size_t)npos * sizeof(float));
    const size_t b_counts = align256(n_counts * sizeof(uint32_t));
    const size_t b_keys = align256((size_t)cells * sizeof(uint32_t));
    const size_t b_ctr = align256(sizeof(cl_counters));
    if ((rc = ensure(h, h->src, b_src)) != CL_OK) return rc;
    if ((rc = ensure(h, h->out, b_counts + b_keys + b_ctr)) != CL_OK) return rc;
    float* d_px = (float*)h->src.p;
    float* d_py = d_px + npos;
    float* d_pz = d_py + npos;
    float* d_pt = d_pz + npos;
    uint32_t* d_counts = (uint32_t*)h->out.p;
    uint32_t* d_keys = (uint32_t*)((char*)h->out.p + b_counts);
    unsigned long long* d_ctr = (unsigned long long*)((char*)h->out.p + b_counts + b_keys);

    cl_records drec;
    memset(&drec, 0, sizeof drec);
    const bool want_rec = records && (records->status || records->idx || records->t || records->bounces);
    if (want_rec && n_photons > 0) {
        const size_t n = (size_t)n_photons;
        const size_t b1 = align256(n), b2 = align256(2 * n), b4 = align256(4 * n);
        if ((rc = ensure(h, h->rec, b1 + b2 + 2 * b4)) != CL_OK) return rc;
        char* base = (char*)h->rec.p;
        if (records->status) drec.status = (uint8_t*)base;
        if (records->idx) drec.idx = (int16_t*)(base + b1);
        if (records->t) drec.t = (float*)(base + b1 + b2);
        if (records->bounces) drec.bounces = (int32_t*)(base + b1 + b2 + b4);
    }

    CK(h, cudaMemcpyAsync(d_px, px, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy px");
    CK(h, cudaMemcpyAsync(d_py, py, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy py");
    CK(h, cudaMemcpyAsync(d_pz, pz, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy pz");
    if (pt) CK(h, cudaMemcpyAsync(d_pt, pt, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy pt");

    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    rc = enqueue_point(h, P, d_px, d_py, d_pz, pt ? d_pt : nullptr, npos, n_photons, pid_offset,
                       d_counts, d_keys, d_ctr, want_rec ? &drec : nullptr, st);
    if (rc != CL_OK) return rc;

    CK(h, cudaMemcpyAsync(counts, d_counts, n_counts * sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "copy counts");
    CK(h, cudaMemcpyAsync(first_ns, d_keys, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, st), "copy first_ns");
    CK(h, cudaMemcpyAsync(counters, d_ctr, sizeof(cl_counters), cudaMemcpyDeviceToHost, st), "copy counters");
    if (want_rec && n_photons > 0) {
        const size_t n = (size_t)n_photons;
        if (records->status) CK(h, cudaMemcpyAsync(records->status, drec.status, n, cudaMemcpyDeviceToHost, st), "copy status");
        if (records->idx) CK(h, cudaMemcpyAsync(records->idx, drec.idx, 2 * n, cudaMemcpyDeviceToHost, st), "copy idx");
        if (records->t) CK(h, cudaMemcpyAsync(records->t, drec.t, 4 * n, cudaMemcpyDeviceToHost, st), "copy t");
        if (records->bounces) CK(h, cudaMemcpyAsync(records->bounces, drec.bounces, 4 * n, cudaMemcpyDeviceToHost, st), "copy bounces");
    }
    return collect(h, st);
}

int cl_run_photons_device(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                          const cl_readout* ro, const cl_time_binning* tb,
                          const float* d_px, const float* d_py, const float* d_pz,
                          const float* d_pt, int32_t npos,
                          int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                          float tau_ns, int32_t max_bounces,
                          uint32_t* d_counts, float* d_first_ns,
                          cl_counters* d_counters, const cl_records* d_records, void* stream)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    if (npos < 1 || !d_px || !d_py || !d_pz) return set_err(h, CL_ERR_ARG, "need npos >= 1 source positions");
    if (n_photons < 0) return set_err(h, CL_ERR_ARG, "n_photons must be >= 0");
    if (!d_counts || !d_first_ns || !d_counters) return set_err(h, CL_ERR_ARG, "null output buffer");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    return enqueue_point(h, P, d_px, d_py, d_pz, d_pt, npos, n_photons, pid_offset, d_counts,
                         (uint32_t*)d_first_ns, (unsigned long long*)d_counters, d_records, st);
}

static int check_segments(cl_handle* h, const int64_t* off, const int32_t* seg, int64_t n_src,
                          int64_t n_seg, int64_t* total)
{
    if (n_src < 1 || n_seg < 1) return set_err(h, CL_ERR_ARG, "need n_src >= 1 and n_segments >= 1");
    if (!off || !seg) return set_err(h, CL_ERR_ARG, "null source offsets or segment ids");
    if (off[0] != 0) return set_err(h, CL_ERR_ARG, "src_offsets[0] must be 0");
    for (int64_t s = 0; s < n_src; ++s) {
        if (off[s + 1] < off[s]) return set_err(h, CL_ERR_ARG, "src_offsets must be non-decreasing");
        if (seg[s] < 0 || seg[s] >= n_seg) return set_err(h, CL_ERR_ARG, "segment id out of range");
        if (s > 0 && seg[s] < seg[s - 1]) return set_err(h, CL_ERR_ARG, "segment ids must be non-decreasing");
    }
    *total = off[n_src];
    return CL_OK;
}

int cl_run_segments(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                    const cl_readout* ro, const cl_time_binning* tb,
                    const float* sx, const float* sy, const float* sz,
                    const float* st_, const int64_t* src_offsets,
                    const int32_t* src_segment, int64_t n_src, int64_t n_segments,
                    uint64_t seed, uint64_t pid_offset,
                    float tau_ns, int32_t max_bounces,
                    uint32_t* maps, float* tmin, int32_t* npe,
                    cl_counters* counters, const cl_records* records)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    int64_t n = 0;
    if ((rc = check_segments(h, src_offsets, src_segment, n_src, n_segments, &n)) != CL_OK) return rc;
    if (!sx || !sy || !sz) return set_err(h, CL_ERR_ARG, "null source positions");
    if (!maps || !tmin || !npe || !counters) return set_err(h, CL_ERR_ARG, "null output buffer");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = h->stream;
    const int cells = ro->grid.nx * ro->grid.ny;
    const size_t total = (size_t)cells * (size_t)n_segments;
    const size_t b_f = align256((size_t)n_src * sizeof(float));
    const size_t b_off = align256((size_t)(n_src + 1) * sizeof(int64_t));
    const size_t b_seg = align256((size_t)n_src * sizeof(int32_t));
    const size_t b_maps = align256(total * sizeof(uint32_t));
    const size_t b_npe = align256((size_t)n_segments * sizeof(int32_t));
    const size_t b_ctr = align256(sizeof(cl_counters));
    if ((rc = ensure(h, h->src, 4 * b_f + b_off + b_seg)) != CL_OK) return rc;
    if ((rc = ensure(h, h->out, 2 * b_maps + b_npe + b_ctr)) != CL_OK) return rc;
    char* sb = (char*)h->src.p;
    float* d_sx = (float*)sb;
    float* d_sy = (float*)(sb + b_f);
    float* d_sz = (float*)(sb + 2 * b_f);
    float* d_st = (float*)(sb + 3 * b_f);
    int64_t* d_off = (int64_t*)(sb + 4 * b_f);
    int32_t* d_seg = (int32_t*)(sb + 4 * b_f + b_off);
    char* ob = (char*)h->out.p;
    uint32_t* d_maps = (uint32_t*)ob;
    uint32_t* d_keys = (uint32_t*)(ob + b_maps);
    int32_t* d_npe = (int32_t*)(ob + 2 * b_maps);
    unsigned long long* d_ctr = (unsigned long long*)(ob + 2 * b_maps + b_npe);

    cl_records drec;
    memset(&drec, 0, sizeof drec);
    const bool want_rec = records && (records->status || records->idx || records->t || records->bounces);
    if (want_rec && n > 0) {
        const size_t m = (size_t)n;
        const size_t b1 = align256(m), b2 = align256(2 * m), b4 = align256(4 * m);
        if ((rc = ensure(h, h->rec, b1 + b2 + 2 * b4)) != CL_OK) return rc;
        char* base = (char*)h->rec.p;
        if (records->status) drec.status = (uint8_t*)base;
        if (records->idx) drec.idx = (int16_t*)(base + b1);
        if (records->t) drec.t = (float*)(base + b1 + b2);
        if (records->bounces) drec.bounces = (int32_t*)(base + b1 + b2 + b4);
    }
    const size_t fs = (size_t)n_src * sizeof(float);
    CK(h, cudaMemcpyAsync(d_sx, sx, fs, cudaMemcpyHostToDevice, st), "copy sx");
    CK(h, cudaMemcpyAsync(d_sy, sy, fs, cudaMemcpyHostToDevice, st), "copy sy");
    CK(h, cudaMemcpyAsync(d_sz, sz, fs, cudaMemcpyHostToDevice, st), "copy sz");
    if (st_) CK(h, cudaMemcpyAsync(d_st, st_, fs, cudaMemcpyHostToDevice, st), "copy st");
    CK(h, cudaMemcpyAsync(d_off, src_offsets, (size_t)(n_src + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st), "copy offsets");
    CK(h, cudaMemcpyAsync(d_seg, src_segment, (size_t)n_src * sizeof(int32_t), cudaMemcpyHostToDevice, st), "copy segments");

    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    rc = enqueue_segments(h, P, d_sx, d_sy, d_sz, st_ ? d_st : nullptr, d_off, d_seg, n_src, n_segments,
                          n, pid_offset, d_maps, d_keys, d_npe, d_ctr, want_rec ? &drec : nullptr, st);
    if (rc != CL_OK) return rc;
    CK(h, cudaMemcpyAsync(maps, d_maps, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "copy maps");
    CK(h, cudaMemcpyAsync(tmin, d_keys, total * sizeof(float), cudaMemcpyDeviceToHost, st), "copy tmin");
    CK(h, cudaMemcpyAsync(npe, d_npe, (size_t)n_segments * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "copy npe");
    CK(h, cudaMemcpyAsync(counters, d_ctr, sizeof(cl_counters), cudaMemcpyDeviceToHost, st), "copy counters");
    if (want_rec && n > 0) {
        const size_t m = (size_t)n;
        if (records->status) CK(h, cudaMemcpyAsync(records->status, drec.status, m, cudaMemcpyDeviceToHost, st), "copy status");
        if (records->idx) CK(h, cudaMemcpyAsync(records->idx, drec.idx, 2 * m, cudaMemcpyDeviceToHost, st), "copy idx");
        if (records->t) CK(h, cudaMemcpyAsync(records->t, drec.t, 4 * m, cudaMemcpyDeviceToHost, st), "copy t");
        if (records->bounces) CK(h, cudaMemcpyAsync(records->bounces, drec.bounces, 4 * m, cudaMemcpyDeviceToHost, st), "copy bounces");
    }
    return collect(h, st);
}

int cl_run_segments_device(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                           const cl_readout* ro, const cl_time_binning* tb,
                           const float* d_sx, const float* d_sy, const float* d_sz,
                           const float* d_st, const int64_t* d_src_offsets,
                           const int32_t* d_src_segment, int64_t n_src, int64_t n_segments,
                           int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                           float tau_ns, int32_t max_bounces,
                           uint32_t* d_maps, float* d_tmin, int32_t* d_npe,
                           cl_counters* d_counters, const cl_records* d_records, void* stream)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    if (n_src < 1 || n_segments < 1) return set_err(h, CL_ERR_ARG, "need n_src >= 1 and n_segments >= 1");
    if (!d_sx || !d_sy || !d_sz || !d_src_offsets || !d_src_segment)
        return set_err(h, CL_ERR_ARG, "null source array");
    if (!d_maps || !d_tmin || !d_npe || !d_counters) return set_err(h, CL_ERR_ARG, "null output buffer");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    const int64_t n = n_photons;
    if (n < 0) return set_err(h, CL_ERR_ARG, "negative photon total");
    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    return enqueue_segments(h, P, d_sx, d_sy, d_sz, d_st, d_src_offsets, d_src_segment, n_src, n_segments,
                            n, pid_offset, d_maps, (uint32_t*)d_tmin, d_npe,
                            (unsigned long long*)d_counters, d_records, st);
}

int cl_run_segments_moments_device(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                                   const cl_readout* ro, const cl_time_binning* tb,
                                   const float* d_sx, const float* d_sy, const float* d_sz,
                                   const float* d_st, const int64_t* d_src_offsets,
                                   const int32_t* d_src_segment, int64_t n_src, int64_t n_segments,
                                   int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                                   float tau_ns, int32_t max_bounces,
                                   uint32_t* d_maps, float* d_tmin, int32_t* d_npe,
                                   cl_counters* d_counters, uint64_t* d_tsum, uint64_t* d_tsum2,
                                   void* stream)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    if (n_src < 1 || n_segments < 1) return set_err(h, CL_ERR_ARG, "need n_src >= 1 and n_segments >= 1");
    if (!d_sx || !d_sy || !d_sz || !d_src_offsets || !d_src_segment)
        return set_err(h, CL_ERR_ARG, "null source array");
    if (!d_maps || !d_tmin || !d_npe || !d_counters || !d_tsum || !d_tsum2)
        return set_err(h, CL_ERR_ARG, "null output buffer");
    if (n_photons < 0) return set_err(h, CL_ERR_ARG, "negative photon total");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    return enqueue_segments(h, P, d_sx, d_sy, d_sz, d_st, d_src_offsets, d_src_segment, n_src, n_segments,
                            n_photons, pid_offset, d_maps, (uint32_t*)d_tmin, d_npe,
                            (unsigned long long*)d_counters, nullptr, st,
                            (unsigned long long*)d_tsum, (unsigned long long*)d_tsum2);
}

int cl_run_events_surrogate_device(cl_handle* h, const cl_box* box, const cl_optical_params* op,
                                   const cl_readout* ro, const cl_time_binning* tb,
                                   const float* d_sx, const float* d_sy, const float* d_sz,
                                   const float* d_st, const int64_t* d_src_offsets,
                                   const int32_t* d_src_segment, int64_t n_src, int64_t n_photons,
                                   uint64_t seed, uint64_t pid_offset, float tau_ns, int32_t max_bounces,
                                   const float* d_site_p, const float* d_site_tmean,
                                   const float* d_site_tsig, const uint8_t* d_site_flag,
                                   const float* d_site_t0, const int64_t* d_site_photons,
                                   const int32_t* d_site_segment, int64_t n_sites, uint64_t sample_seed,
                                   int64_t n_segments, uint32_t* d_maps, float* d_tmin, int32_t* d_npe,
                                   cl_counters* d_counters, uint64_t* d_sampled, void* stream)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    int rc = check_params(h, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return rc;
    if (n_segments < 1) return set_err(h, CL_ERR_ARG, "need n_segments >= 1");
    if (n_src < 0 || n_sites < 0 || n_photons < 0) return set_err(h, CL_ERR_ARG, "negative size");
    if (n_src == 0 && n_photons != 0) return set_err(h, CL_ERR_ARG, "photons without Monte Carlo sources");
    if (n_src > 0 && (!d_sx || !d_sy || !d_sz || !d_src_offsets || !d_src_segment))
        return set_err(h, CL_ERR_ARG, "null source array");
    if (n_sites > 0 && (!d_site_p || !d_site_tmean || !d_site_tsig || !d_site_t0 || !d_site_photons ||
                        !d_site_segment))
        return set_err(h, CL_ERR_ARG, "null surrogate site array");
    if (!d_maps || !d_tmin || !d_npe || !d_counters) return set_err(h, CL_ERR_ARG, "null output buffer");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    SurSampleArgs sa;
    memset(&sa, 0, sizeof sa);
    sa.p = d_site_p; sa.tmean = d_site_tmean; sa.tsig = d_site_tsig; sa.flag = d_site_flag;
    sa.t0 = d_site_t0; sa.photons = d_site_photons; sa.seg = d_site_segment; sa.n = n_sites;
    sa.n_seg = n_segments;
    sa.cells = ro->grid.nx * ro->grid.ny;
    sa.k0 = (uint32_t)sample_seed; sa.k1 = (uint32_t)(sample_seed >> 32);
    sa.tau = tau_ns;
    sa.stats = (unsigned long long*)d_sampled;
    if (d_sampled) CK(h, cudaMemsetAsync(d_sampled, 0, 2 * sizeof(uint64_t), st), "zero sampler stats");
    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    return enqueue_segments(h, P, d_sx, d_sy, d_sz, d_st, d_src_offsets, d_src_segment, n_src, n_segments,
                            n_photons, pid_offset, d_maps, (uint32_t*)d_tmin, d_npe,
                            (unsigned long long*)d_counters, nullptr, st, nullptr, nullptr, &sa);
}

int cl_sync(cl_handle* h, void* stream)
{
    if (!h) return CL_ERR_STATE;
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    return collect(h, stream ? (cudaStream_t)stream : h->stream);
}

int cl_debug_eval(cl_handle* h, int fn, const void* in, void* out, int64_t n, uint64_t seed, int32_t n_per)
{
    if (!h) return CL_ERR_STATE;
    h->err[0] = 0;
    if (n < 0 || !out || (fn != 4 && fn != 6 && !in)) return set_err(h, CL_ERR_ARG, "bad debug arguments");
    if (fn < 0 || fn > 6) return set_err(h, CL_ERR_ARG, "unknown debug function");
    if (fn == 4 && n_per < 1) return set_err(h, CL_ERR_ARG, "n_per must be >= 1");
    CK(h, cudaSetDevice(h->device), "cudaSetDevice");
    cudaStream_t st = h->stream;
    if (fn == 6) {
        // the handle's table of the logs of the uniforms (2^24 floats)
        if (!h->logtab.p) return set_err(h, CL_ERR_STATE, "this handle has no log table");
        if (n > (1 << 24)) return set_err(h, CL_ERR_ARG, "the log table has 2^24 entries");
        CK(h, cudaMemcpyAsync(out, h->logtab.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, st), "copy table");
        CK(h, cudaStreamSynchronize(st), "stream synchronize");
        return CL_OK;
    }
    size_t in_b = 0, out_b = 0;
    if (fn <= 2) { in_b = 4 * (size_t)n; out_b = 4 * (size_t)n; }
    else if (fn == 3 || fn == 5) { in_b = 16 * (size_t)n; out_b = 16 * (size_t)n; }
    else { out_b = 4 * (size_t)n * (size_t)n_per; }
    int rc = ensure(h, h->dbg, align256(in_b) + align256(out_b) + 256);
    if (rc != CL_OK) return rc;
    char* din = (char*)h->dbg.p;
    char* dout = din + align256(in_b);
    if (in_b) CK(h, cudaMemcpyAsync(din, in, in_b, cudaMemcpyHostToDevice, st), "copy in");
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16));
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    if (n > 0) {
        if (fn <= 2) debug_math_kernel<<<grid, 256, 0, st>>>(fn, (const float*)din, (float*)dout, n);
        else if (fn == 3 || fn == 5)
            debug_philox_kernel<<<grid, 256, 0, st>>>(fn == 5, (const uint32_t*)din, (uint32_t*)dout, n, k0, k1);
        else debug_randu_kernel<<<grid, 256, 0, st>>>((float*)dout, n, n_per, k0, k1);
        CK(h, cudaGetLastError(), "debug kernel launch");
    }
    if (out_b) CK(h, cudaMemcpyAsync(out, dout, out_b, cudaMemcpyDeviceToHost, st), "copy out");
    CK(h, cudaStreamSynchronize(st), "stream synchronize");
    return CL_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free entry point (cl_run_photons_noalloc).
//
// For callers that cannot let a library call cudaMalloc (device memory owned
// by a pool/caching allocator or a fixed budget; loops where cudaMalloc or
// cudaFree would synchronise the device).  All device memory it touches is
// the file-scope array below, CL_NOALLOC_SCRATCH_BYTES long, which each GPU
// that loads this library holds until the process exits.  Every call reuses
// (and overwrites) the whole array: calls that overlap on the GPU race.
// ===========================================================================
static __device__ __align__(256) unsigned char g_noalloc_scratch[CL_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
struct NoallocDevice {
    bool ready = false;
    unsigned char* base = nullptr;   // device address of g_noalloc_scratch on this device
    int num_sms = 0;
    int max_smem_optin = 0;
    int max_smem_per_sm = 0;
};
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

// Once per device, with that device current: look up the array's device
// address (host code cannot use the symbol itself as a device pointer) and
// the launch limits.  Allocates nothing.
int noalloc_setup(int dev, NoallocDevice** out)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoallocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&d.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&d.max_smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            snprintf(g_create_err, sizeof g_create_err, "cl_run_photons_noalloc: set-up on device %d: %s",
                     dev, cudaGetErrorString(e));
            return CL_ERR_CUDA;
        }
        set_kernel_attrs<0, false, true>(d.max_smem_optin);
        set_kernel_attrs<0, false, false>(d.max_smem_optin);
        cudaGetLastError();
        d.base = (unsigned char*)p;
        d.ready = true;
    }
    *out = &d;
    return CL_OK;
}
}  // namespace

extern "C" int cl_run_photons_noalloc(const cl_box* box, const cl_optical_params* op,
                                      const cl_readout* ro, const cl_time_binning* tb,
                                      const float* px, const float* py, const float* pz,
                                      const float* pt, int32_t npos,
                                      int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                                      float tau_ns, int32_t max_bounces,
                                      uint32_t* counts, float* first_ns, cl_counters* counters,
                                      void* stream)
{
    g_create_err[0] = 0;
    // A stack handle carries the launch settings and collects error messages;
    // its scratch words point into the static array.  Nothing is allocated.
    cl_handle tmp;
    auto fail = [&](int rc) {
        snprintf(g_create_err, sizeof g_create_err, "cl_run_photons_noalloc: %s", tmp.err);
        return rc;
    };
    int rc = check_params(&tmp, box, op, ro, tb, tau_ns, max_bounces);
    if (rc != CL_OK) return fail(rc);
    if (npos < 1 || !px || !py || !pz) return fail(set_err(&tmp, CL_ERR_ARG, "need npos >= 1 source positions"));
    if (n_photons < 0) return fail(set_err(&tmp, CL_ERR_ARG, "n_photons must be >= 0"));
    if (!counts || !first_ns || !counters) return fail(set_err(&tmp, CL_ERR_ARG, "null output buffer"));

    const int cells = ro->grid.nx * ro->grid.ny;
    const size_t n_counts = (size_t)cells * (size_t)(tb->nbins + 1);
    const size_t b_words = 256, b_ctr = 256;
    const size_t b_counts = align256(n_counts * sizeof(uint32_t));
    const size_t b_keys = align256((size_t)cells * sizeof(uint32_t));
    const size_t b_src = align256((size_t)npos * sizeof(float));
    const size_t need = b_words + b_ctr + b_counts + b_keys + 4 * b_src;
    if (need > (size_t)CL_NOALLOC_SCRATCH_BYTES)
        return fail(set_err(&tmp, CL_ERR_ARG,
                            "staged data needs %zu bytes (npos %d, %d cells x %d bins) but the "
                            "static device array holds %u bytes",
                            need, (int)npos, cells, tb->nbins + 1, (unsigned)CL_NOALLOC_SCRATCH_BYTES));

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        cudaGetLastError();
        return fail(set_err(&tmp, CL_ERR_CUDA, "no current CUDA device (%s)",
                            e != cudaSuccess ? cudaGetErrorString(e) : "device index out of range"));
    }
    NoallocDevice* nd = nullptr;
    if ((rc = noalloc_setup(dev, &nd)) != CL_OK) return rc;

    tmp.device = dev;
    tmp.num_sms = nd->num_sms;
    tmp.max_smem_optin = nd->max_smem_optin;
    tmp.max_smem_per_sm = nd->max_smem_per_sm;
    tmp.scratch.p = nd->base;                 // queue / steps / done / err words
    tmp.scratch.cap = b_words;
    unsigned char* base = nd->base;
    unsigned long long* d_ctr = (unsigned long long*)(base + b_words);
    uint32_t* d_counts = (uint32_t*)(base + b_words + b_ctr);
    uint32_t* d_keys = (uint32_t*)(base + b_words + b_ctr + b_counts);
    float* d_px = (float*)(base + b_words + b_ctr + b_counts + b_keys);
    float* d_py = (float*)((unsigned char*)d_px + b_src);
    float* d_pz = (float*)((unsigned char*)d_py + b_src);
    float* d_pt = (float*)((unsigned char*)d_pz + b_src);
    cudaStream_t st = (cudaStream_t)stream;

#define NK(call, what)                                                        \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return fail(cuda_fail(&tmp, e_, (what)));      \
    } while (0)
    NK(cudaMemcpyAsync(d_px, px, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy px");
    NK(cudaMemcpyAsync(d_py, py, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy py");
    NK(cudaMemcpyAsync(d_pz, pz, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy pz");
    if (pt) NK(cudaMemcpyAsync(d_pt, pt, npos * sizeof(float), cudaMemcpyHostToDevice, st), "copy pt");

    // The init kernel clears the counts, keys, counters and queue words left
    // by the previous call before the transport kernel runs.
    const Physics P = make_physics(box, op, ro, tb, tau_ns, max_bounces, seed);
    rc = enqueue_point(&tmp, P, d_px, d_py, d_pz, pt ? d_pt : nullptr, npos, n_photons, pid_offset,
                       d_counts, d_keys, d_ctr, nullptr, st);
    if (rc != CL_OK) return fail(rc);
    NK(cudaMemcpyAsync(counts, d_counts, n_counts * sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "copy counts");
    NK(cudaMemcpyAsync(first_ns, d_keys, (size_t)cells * sizeof(float), cudaMemcpyDeviceToHost, st), "copy first_ns");
    NK(cudaMemcpyAsync(counters, d_ctr, sizeof(cl_counters), cudaMemcpyDeviceToHost, st), "copy counters");
#undef NK
    rc = collect(&tmp, st);
    if (rc != CL_OK) return fail(rc);
    return CL_OK;
}
