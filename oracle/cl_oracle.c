/*
 * cl_oracle.c — CPU restatement of CryspLight's optical-photon transport.
 *
 * TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline; never shipped or
 * called by the product).  Every function cites the reference lines it
 * follows.  Build with -ffp-contract=off and without -ffast-math: Julia does
 * not fuse multiply-adds and evaluates left to right, so every expression
 * below keeps the reference's association, e.g. (2f0*Float32(pi))*u and
 * (-tau)*log(u); `x^2` on a literal exponent is Julia's literal_pow, i.e. x*x.
 */
#include "cl_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* Reference-operation counting (built only into the analysis variant with
 * -DOR_COUNT_OPS): OPS(n) adds the number of Float32/integer arithmetic
 * operations (+ - * / sqrt, and log/sin/cos as one each; comparisons and
 * selects not counted) that the reference's expression at that point
 * performs.  Used to state the algorithmic work per photon-step. */
#ifdef OR_COUNT_OPS
static __thread uint64_t or_ops_counter;
#define OPS(n) (or_ops_counter += (uint64_t)(n))
uint64_t or_ops_read(void) { return or_ops_counter; }
void or_ops_reset(void) { or_ops_counter = 0; }
#else
#define OPS(n) ((void)0)
uint64_t or_ops_read(void) { return 0; }
void or_ops_reset(void) {}
#endif

/* ------------------------------------------------------------------------ */
/* Philox4x32-10, src/philox.jl:5-28                                         */
/* ------------------------------------------------------------------------ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    OPS(10 * 6 + 9 * 2);
    for (int r = 1; r <= 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        if (r < 10) {
            k0 += PHILOX_W0;
            k1 += PHILOX_W1;
        }
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* PhiloxStream(seed, photon_id), src/philox.jl:43-48: i = 5 so the first
 * draw generates block 0. */
void or_stream_init(or_stream* s, uint64_t seed, uint64_t photon_id)
{
    s->key[0] = (uint32_t)seed;
    s->key[1] = (uint32_t)(seed >> 32);
    s->id_lo = (uint32_t)photon_id;
    s->id_hi = (uint32_t)(photon_id >> 32);
    s->block = 0;
    s->buf[0] = s->buf[1] = s->buf[2] = s->buf[3] = 0;
    s->i = 5;
}

/* next_u32!, src/philox.jl:50-59 (1-based i in the reference). */
uint32_t or_next_u32(or_stream* s)
{
    if (s->i > 4) {
        uint32_t ctr[4] = {s->id_lo, s->id_hi, s->block, 0u};
        or_philox4x32(ctr, s->key, s->buf);
        s->block += 1u;
        s->i = 1;
    }
    uint32_t x = s->buf[s->i - 1];
    s->i += 1;
    return x;
}

/* randu, src/philox.jl:62: ((x >>> 8) + 1.0f0) * Float32(exp2(-24)). */
float or_randu(or_stream* s)
{
    uint32_t x = or_next_u32(s);
    OPS(4);
    float v = (float)(x >> 8) + 1.0f;
    return v * 0x1p-24f;
}

/* ------------------------------------------------------------------------ */
/* Elementary functions: Float64 evaluation rounded once to Float32.          */
/* ------------------------------------------------------------------------ */
float or_logf(float x) { OPS(1); return (float)log((double)x); }
float or_sinf(float x) { OPS(1); return (float)sin((double)x); }
float or_cosf(float x) { OPS(1); return (float)cos((double)x); }

static const float TWO_PI_F = 2.0f * 3.14159265358979323846f;  /* 2f0*Float32(pi), exact */

/* ------------------------------------------------------------------------ */
/* Geometry, src/geometry.jl:6-32                                            */
/* ------------------------------------------------------------------------ */
enum { FACE_XP = 1, FACE_XM = 2, FACE_YP = 3, FACE_YM = 4, FACE_BACK = 5, FACE_FRONT = 6 };

int32_t or_wall_hit(float x, float y, float z, float ux, float uy, float uz,
                    const cl_box* box, float* d)
{
    const float Lx = box->L[0], Ly = box->L[1], Lz = box->L[2];
    OPS(2 * ((ux != 0.0f) + (uy != 0.0f) + (uz != 0.0f)));
    float dx = ux > 0.0f ? (Lx - x) / ux : (ux < 0.0f ? (-x) / ux : INFINITY);
    float dy = uy > 0.0f ? (Ly - y) / uy : (uy < 0.0f ? (-y) / uy : INFINITY);
    float dz = uz > 0.0f ? (Lz - z) / uz : (uz < 0.0f ? (-z) / uz : INFINITY);
    if (dx <= dy && dx <= dz) {
        *d = dx;
        return ux > 0.0f ? FACE_XP : FACE_XM;
    } else if (dy <= dz) {
        *d = dy;
        return uy > 0.0f ? FACE_YP : FACE_YM;
    } else {
        *d = dz;
        return uz > 0.0f ? FACE_BACK : FACE_FRONT;
    }
}

/* ------------------------------------------------------------------------ */
/* Optics, src/optics.jl                                                     */
/* ------------------------------------------------------------------------ */

/* fresnel, src/optics.jl:10-19. */
int or_fresnel(float n1, float n2, float cosi, float* R)
{
    float q = n1 / n2;
    float sin2t = (q * q) * (1.0f - cosi * cosi);
    OPS(5);
    if (sin2t >= 1.0f) {
        *R = 1.0f;
        return 1;
    }
    float cost = sqrtf(1.0f - sin2t);
    OPS(2 + 7 + 7 + 4);
    float a = (n1 * cosi - n2 * cost) / (n1 * cosi + n2 * cost);
    float b = (n1 * cost - n2 * cosi) / (n1 * cost + n2 * cosi);
    float rs = a * a;
    float rp = b * b;
    *R = 0.5f * (rs + rp);
    return 0;
}

/* face_axis, src/optics.jl:22 (1, 2, 3). */
static inline int face_axis(int32_t face) { return face <= 2 ? 1 : (face <= 4 ? 2 : 3); }

/* specular, src/optics.jl:25-28. */
static inline void specular(float u[3], int32_t face)
{
    int a = face_axis(face);
    u[a - 1] = -u[a - 1];
}

/* gaussian, src/optics.jl:38-39: first draw feeds log, second cos. */
float or_gaussian(or_stream* s)
{
    float u1 = or_randu(s);
    float l = or_logf(u1);
    float u2 = or_randu(s);
    OPS(4);
    return sqrtf(-2.0f * l) * or_cosf(TWO_PI_F * u2);
}

/* surface_interact, src/optics.jl:49-81. */
int or_surface_interact(or_stream* s, const float u[3], int32_t face,
                        float n_crystal, float sigma_alpha, float v[3])
{
    const float ux = u[0], uy = u[1], uz = u[2];
    const int a = face_axis(face);
    const float sgn = (face == FACE_XP || face == FACE_YP || face == FACE_BACK) ? 1.0f : -1.0f;
    const float Nx = a == 1 ? sgn : 0.0f;
    const float Ny = a == 2 ? sgn : 0.0f;
    const float Nz = a == 3 ? sgn : 0.0f;
    for (int tries = 0; tries < 20; ++tries) {
        float alpha = sigma_alpha * fabsf(or_gaussian(s));
        OPS(2);
        if (alpha >= 1.2f) continue;
        float ca = or_cosf(alpha), sa = or_sinf(alpha);
        float phi = TWO_PI_F * or_randu(s);
        float b = sa * or_cosf(phi), c = sa * or_sinf(phi);
        OPS(1 + 2 + 1 + 5);  /* phi, b, c, ca*sgn, cosi */
        float Nfx = a == 1 ? ca * sgn : b;
        float Nfy = a == 2 ? ca * sgn : (a == 1 ? b : c);
        float Nfz = a == 3 ? ca * sgn : c;
        float cosi = ux * Nfx + uy * Nfy + uz * Nfz;
        if (cosi <= 0.0f) continue;
        float R;
        int tir = or_fresnel(n_crystal, 1.0f, cosi, &R);
        if (tir || or_randu(s) < R) {
            OPS(7 + 5);  /* reflection, inside test */
            float rx = ux - (2.0f * cosi) * Nfx;
            float ry = uy - (2.0f * cosi) * Nfy;
            float rz = uz - (2.0f * cosi) * Nfz;
            if (rx * Nx + ry * Ny + rz * Nz < 0.0f) {
                v[0] = rx; v[1] = ry; v[2] = rz;
                return 0;
            }
        } else {
            v[0] = ux; v[1] = uy; v[2] = uz;
            return 1;
        }
    }
    v[0] = ux; v[1] = uy; v[2] = uz;
    specular(v, face);
    return 0;
}

/* rayleigh_dir, src/optics.jl:87-112. */
void or_rayleigh_dir(or_stream* s, const float u[3], float v[3])
{
    const float ux = u[0], uy = u[1], uz = u[2];
    float mu;
    for (;;) {
        mu = 1.0f - 2.0f * or_randu(s);
        OPS(5);
        if (2.0f * or_randu(s) <= 1.0f + mu * mu) break;
    }
    float st = sqrtf(fmaxf(0.0f, 1.0f - mu * mu));
    float phi = TWO_PI_F * or_randu(s);
    float cb = st * or_cosf(phi), sb = st * or_sinf(phi);
    OPS(4 + 1 + 2 + 7 + 9 + 15 + 10);  /* st, phi, cb/sb, t1, t2, v, normalise */
    float t1x, t1y, t1z, inv;
    if (fabsf(uz) < 0.9f) {
        inv = 1.0f / sqrtf(ux * ux + uy * uy);
        t1x = -uy * inv; t1y = ux * inv; t1z = 0.0f;
    } else {
        inv = 1.0f / sqrtf(uy * uy + uz * uz);
        t1x = 0.0f; t1y = -uz * inv; t1z = uy * inv;
    }
    float t2x = uy * t1z - uz * t1y;
    float t2y = uz * t1x - ux * t1z;
    float t2z = ux * t1y - uy * t1x;
    float vx = mu * ux + cb * t1x + sb * t2x;
    float vy = mu * uy + cb * t1y + sb * t2y;
    float vz = mu * uz + cb * t1z + sb * t2z;
    inv = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
    v[0] = vx * inv; v[1] = vy * inv; v[2] = vz * inv;
}

/* lambertian_dir, src/optics.jl:118-138. */
void or_lambertian_dir(or_stream* s, int32_t face, float u[3])
{
    float ct = sqrtf(or_randu(s));
    float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float phi = TWO_PI_F * or_randu(s);
    OPS(1 + 4 + 1 + 2 + 1);  /* sqrt, st, phi, a/b, inward sign */
    float a = st * or_cosf(phi);
    float b = st * or_sinf(phi);
    switch (face) {
    case FACE_XP: u[0] = -ct; u[1] = a; u[2] = b; break;
    case FACE_XM: u[0] = ct;  u[1] = a; u[2] = b; break;
    case FACE_YP: u[0] = a; u[1] = -ct; u[2] = b; break;
    case FACE_YM: u[0] = a; u[1] = ct;  u[2] = b; break;
    case FACE_BACK: u[0] = a; u[1] = b; u[2] = -ct; break;
    default:        u[0] = a; u[1] = b; u[2] = ct;  break;
    }
}

/* ------------------------------------------------------------------------ */
/* Generation, src/generation.jl:4-13                                        */
/* ------------------------------------------------------------------------ */
void or_isotropic_dir(or_stream* s, float u[3])
{
    float uz = 1.0f - 2.0f * or_randu(s);
    float r = sqrtf(fmaxf(0.0f, 1.0f - uz * uz));
    OPS(2 + 4 + 1 + 2);
    float phi = TWO_PI_F * or_randu(s);
    u[0] = r * or_cosf(phi);
    u[1] = r * or_sinf(phi);
    u[2] = uz;
}

float or_emission_time(or_stream* s, float tau_ns)
{
    if (tau_ns > 0.0f) OPS(1);
    return tau_ns > 0.0f ? (-tau_ns) * or_logf(or_randu(s)) : 0.0f;
}

/* ------------------------------------------------------------------------ */
/* Transport, src/transport.jl:96-234                                        */
/* ------------------------------------------------------------------------ */
static const float C_MM_NS = 299.792458f;

/* Counts the aperture test's operations; always true. */
static inline int count_disc_ops(const cl_readout* ro)
{
    if (ro->disc) OPS(5);
    return 1;
}

static inline int32_t trunc_i32(float v) { return (int32_t)v; }   /* unsafe_trunc */

/* SiPM cell (1-based ii, jj) of a detection, src/transport.jl:98-99. */
static inline void sipm_cell(const cl_sipm_grid* g, float x, float y, int32_t* ii, int32_t* jj)
{
    int32_t i = 1 + trunc_i32(x / g->pitch_mm);
    int32_t j = 1 + trunc_i32(y / g->pitch_mm);
    *ii = i < g->nx ? i : g->nx;
    *jj = j < g->ny ? j : g->ny;
}

/* Time bin (1-based, nbins+1 = overflow), src/transport.jl:100-101. */
static inline int32_t time_bin(const cl_time_binning* tb, float t)
{
    float q = t / tb->bin_ns;
    if (!(q < (float)tb->nbins)) return tb->nbins + 1;   /* 1 + trunc(q) > nbins */
    int32_t b = 1 + trunc_i32(q);
    return b < 1 ? 1 : b;  /* t < 0 is outside the reference's domain (BoundsError) */
}

/* record_detection!, src/transport.jl:96-108. */
static void record_detection(or_acc* acc, const cl_sipm_grid* g, const cl_time_binning* tb,
                             float x, float y, float t, int32_t bounces)
{
    int32_t i, j;
    sipm_cell(g, x, y, &i, &j);
    int32_t bin = time_bin(tb, t);
    size_t cell = (size_t)(i - 1) + (size_t)acc->nx * (size_t)(j - 1);
    acc->counts[cell + (size_t)acc->nx * acc->ny * (size_t)(bin - 1)] += 1u;
    if (t < acc->first_ns[cell]) acc->first_ns[cell] = t;
    acc->c.ndet += 1;
    acc->c.sum_bounces_det += bounces;
}

int32_t or_propagate_photon(or_acc* acc, const cl_box* box,
                            const cl_optical_params* op, const cl_readout* ro,
                            const cl_time_binning* tb, or_stream* s,
                            float x, float y, float z,
                            float ux, float uy, float uz, float t0,
                            int32_t max_bounces, or_photon* out)
{
    float t = t0;
    const float inv_v = op->n_crystal / C_MM_NS;
    int32_t bounces = 0, nscat = 0, steps = 0;
    int16_t idx = 0;
    int32_t status;
    float u[3] = {ux, uy, uz};
    for (;;) {
        steps += 1;
        float d;
        int32_t face = or_wall_hit(x, y, z, u[0], u[1], u[2], box, &d);
        float d_abs = isfinite(op->abs_len_mm) ? (-op->abs_len_mm) * or_logf(or_randu(s)) : INFINITY;
        float d_ray = isfinite(op->rayleigh_mm) ? (-op->rayleigh_mm) * or_logf(or_randu(s)) : INFINITY;
        OPS(isfinite(op->abs_len_mm) + isfinite(op->rayleigh_mm));
        if (d_abs < d && d_abs <= d_ray) {
            if (acc) acc->c.nabs_bulk += 1;
            status = CL_STATUS_ABS_BULK;
            break;
        } else if (d_ray < d) {
            x += d_ray * u[0]; y += d_ray * u[1]; z += d_ray * u[2];
            t += d_ray * inv_v;
            OPS(8 + 2);  /* advance; nscat, bounces */
            float v[3];
            or_rayleigh_dir(s, u, v);
            u[0] = v[0]; u[1] = v[1]; u[2] = v[2];
            if (acc) acc->c.nscat += 1;
            nscat += 1;
            bounces += 1;
            if (bounces >= max_bounces) {
                if (acc) acc->c.ncap += 1;
                status = CL_STATUS_CAP;
                break;
            }
            continue;
        }
        /* advance to the wall; clamp, then snap the hit axis (src/transport.jl:146-157) */
        float nx_ = x + d * u[0], ny_ = y + d * u[1], nz_ = z + d * u[2];
        x = nx_ > box->L[0] ? box->L[0] : (nx_ < 0.0f ? 0.0f : nx_);
        y = ny_ > box->L[1] ? box->L[1] : (ny_ < 0.0f ? 0.0f : ny_);
        z = nz_ > box->L[2] ? box->L[2] : (nz_ < 0.0f ? 0.0f : nz_);
        int a = face_axis(face);
        if (a == 1)      x = face == FACE_XP ? box->L[0] : 0.0f;
        else if (a == 2) y = face == FACE_YP ? box->L[1] : 0.0f;
        else             z = face == FACE_BACK ? box->L[2] : 0.0f;
        t += d * inv_v;
        float cosi = a == 1 ? fabsf(u[0]) : (a == 2 ? fabsf(u[1]) : fabsf(u[2]));
        OPS(6 + 2 + 1 + 1);  /* advance, time, |u|, bounce count */

        if (face == FACE_BACK || (ro->two_sided && face == FACE_FRONT)) {
            /* readout face, src/transport.jl:161-185 */
            float R;
            int tir = or_fresnel(op->n_crystal, op->n_coupling, cosi, &R);
            if (tir || or_randu(s) < R) {
                specular(u, face);
            } else if (count_disc_ops(ro) &&
                       (!ro->disc ||
                       (x - ro->cx) * (x - ro->cx) + (y - ro->cy) * (y - ro->cy) <= ro->r2)) {
                if (or_randu(s) <= op->pde) {
                    int32_t ii, jj;
                    sipm_cell(&ro->grid, x, y, &ii, &jj);
                    int32_t lin = (jj - 1) * ro->grid.nx + ii;
                    OPS(2 * 2 + 3);  /* cell i, j; linear index */
                    idx = (int16_t)(face == FACE_FRONT ? -lin : lin);
                    if (acc) {
                        record_detection(acc, &ro->grid, tb, x, y, t, bounces);
                        if (face == FACE_FRONT) acc->c.ndet_front += 1;
                    }
                    status = CL_STATUS_DETECTED;
                    break;
                } else {
                    if (acc) acc->c.nabs_sipm += 1;
                    status = CL_STATUS_ABS_SIPM;
                    break;
                }
            } else if (or_randu(s) <= ro->sur_R) {
                if (ro->sur_specular) specular(u, face);
                else or_lambertian_dir(s, face, u);
            } else {
                if (acc) acc->c.nabs_sur += 1;
                status = CL_STATUS_ABS_SUR;
                break;
            }
        } else if (!op->air_gap) {
            /* front-painted wrap, src/transport.jl:186-198 */
            if (or_randu(s) <= op->wrap_R) {
                if (op->wrap_specular) specular(u, face);
                else or_lambertian_dir(s, face, u);
            } else {
                if (acc) acc->c.nabs_wall += 1;
                status = CL_STATUS_ABS_WALL;
                break;
            }
        } else {
            /* back-painted wrap, src/transport.jl:199-226 */
            int transmitted = 0;
            if (op->sigma_alpha > 0.0f) {
                float v[3];
                transmitted = or_surface_interact(s, u, face, op->n_crystal, op->sigma_alpha, v);
                u[0] = v[0]; u[1] = v[1]; u[2] = v[2];
            } else {
                float R;
                int tir = or_fresnel(op->n_crystal, 1.0f, cosi, &R);
                if (tir || or_randu(s) < R) specular(u, face);
                else transmitted = 1;
            }
            if (transmitted) {
                if (or_randu(s) <= op->wrap_R) {
                    if (op->wrap_specular) specular(u, face);
                    else or_lambertian_dir(s, face, u);
                } else {
                    if (acc) acc->c.nabs_wall += 1;
                    status = CL_STATUS_ABS_WALL;
                    break;
                }
            }
        }
        bounces += 1;
        if (bounces >= max_bounces) {
            if (acc) acc->c.ncap += 1;
            status = CL_STATUS_CAP;
            break;
        }
    }
    if (out) {
        out->status = status;
        out->idx = idx;
        out->t = t;
        out->bounces = bounces;
        out->nscat = nscat;
        out->steps = steps;
    }
    return status;
}

/* ------------------------------------------------------------------------ */
/* Accumulator helpers                                                       */
/* ------------------------------------------------------------------------ */
static int acc_alloc(or_acc* a, const cl_readout* ro, const cl_time_binning* tb)
{
    a->nx = ro->grid.nx; a->ny = ro->grid.ny; a->nbins = tb->nbins;
    size_t ncell = (size_t)a->nx * a->ny;
    a->counts = (uint32_t*)calloc(ncell * (size_t)(a->nbins + 1), sizeof(uint32_t));
    a->first_ns = (float*)malloc(ncell * sizeof(float));
    memset(&a->c, 0, sizeof a->c);
    if (!a->counts || !a->first_ns) return -1;
    for (size_t i = 0; i < ncell; ++i) a->first_ns[i] = INFINITY;
    return 0;
}

static void acc_free(or_acc* a) { free(a->counts); free(a->first_ns); }

/* merge!, src/transport.jl:82-91. */
static void acc_merge(or_acc* a, const or_acc* b)
{
    size_t ncell = (size_t)a->nx * a->ny, n = ncell * (size_t)(a->nbins + 1);
    for (size_t i = 0; i < n; ++i) a->counts[i] += b->counts[i];
    for (size_t i = 0; i < ncell; ++i)
        a->first_ns[i] = b->first_ns[i] < a->first_ns[i] ? b->first_ns[i] : a->first_ns[i];
    a->c.ndet += b->c.ndet; a->c.ndet_front += b->c.ndet_front;
    a->c.nabs_bulk += b->c.nabs_bulk; a->c.nabs_wall += b->c.nabs_wall;
    a->c.nabs_sipm += b->c.nabs_sipm; a->c.ncap += b->c.ncap; a->c.nabs_sur += b->c.nabs_sur;
    a->c.nscat += b->c.nscat;
    a->c.sum_bounces_det += b->c.sum_bounces_det;
}

static int clamp_threads(int nthreads, int64_t n)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    if (n < nthreads) nthreads = n > 0 ? (int)n : 1;
    return nthreads;
}

/* ------------------------------------------------------------------------ */
/* run_photons!, src/transport.jl:245-273                                    */
/* ------------------------------------------------------------------------ */
typedef struct rp_job {
    const cl_box* box; const cl_optical_params* op; const cl_readout* ro;
    const cl_time_binning* tb;
    const float *px, *py, *pz; int32_t npos;
    int64_t n; uint64_t seed; float tau; int32_t maxb;
    int tid, nt;
    or_acc acc;
} rp_job;

static void* rp_worker(void* arg)
{
    rp_job* j = (rp_job*)arg;
    /* pid in tid:nt:n_photons (1-based tid) */
    for (int64_t pid = j->tid + 1; pid <= j->n; pid += j->nt) {
        or_stream s;
        or_stream_init(&s, j->seed, (uint64_t)pid);
        int64_t p = (pid - 1) % j->npos;
        float u[3];
        or_isotropic_dir(&s, u);
        float t0 = or_emission_time(&s, j->tau);
        or_propagate_photon(&j->acc, j->box, j->op, j->ro, j->tb, &s,
                            j->px[p], j->py[p], j->pz[p], u[0], u[1], u[2], t0, j->maxb, NULL);
    }
    return NULL;
}

int or_run_photons(const cl_box* box, const cl_optical_params* op,
                   const cl_readout* ro, const cl_time_binning* tb,
                   const float* px, const float* py, const float* pz, int32_t npos,
                   int64_t n_photons, uint64_t seed, float tau_ns,
                   int32_t max_bounces, int nthreads,
                   uint32_t* counts, float* first_ns, cl_counters* counters)
{
    if (npos < 1 || n_photons < 0) return -1;
    int nt = clamp_threads(nthreads, n_photons);
    rp_job* jobs = (rp_job*)calloc((size_t)nt, sizeof(rp_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nt, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1; }
    int rc = 0;
    for (int t = 0; t < nt; ++t) {
        rp_job* j = &jobs[t];
        j->box = box; j->op = op; j->ro = ro; j->tb = tb;
        j->px = px; j->py = py; j->pz = pz; j->npos = npos;
        j->n = n_photons; j->seed = seed; j->tau = tau_ns; j->maxb = max_bounces;
        j->tid = t; j->nt = nt;
        if (acc_alloc(&j->acc, ro, tb)) rc = -1;
    }
    if (rc == 0) {
        for (int t = 1; t < nt; ++t) pthread_create(&th[t], NULL, rp_worker, &jobs[t]);
        rp_worker(&jobs[0]);
        for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
        for (int t = 1; t < nt; ++t) acc_merge(&jobs[0].acc, &jobs[t].acc);
        size_t ncell = (size_t)ro->grid.nx * ro->grid.ny;
        memcpy(counts, jobs[0].acc.counts, ncell * (size_t)(tb->nbins + 1) * sizeof(uint32_t));
        memcpy(first_ns, jobs[0].acc.first_ns, ncell * sizeof(float));
        *counters = jobs[0].acc.c;
    }
    for (int t = 0; t < nt; ++t) acc_free(&jobs[t].acc);
    free(jobs); free(th);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* transport_kernel! records + run_photons_ka! reduction, src/kernel.jl       */
/* ------------------------------------------------------------------------ */

/* One photon of the kernel twin (src/kernel.jl:162-183): stream keyed by pid,
 * starting point and time offset from its source. */
static void ka_photon(const cl_box* box, const cl_optical_params* op, const cl_readout* ro,
                      const cl_time_binning* tb, uint64_t seed, uint64_t pid,
                      float x, float y, float z, float pt, float tau, int32_t maxb,
                      or_photon* ph)
{
    or_stream s;
    or_stream_init(&s, seed, pid);
    float u[3];
    or_isotropic_dir(&s, u);
    float t = pt;
    if (tau > 0.0f) t += (-tau) * or_logf(or_randu(&s));
    or_propagate_photon(NULL, box, op, ro, tb, &s, x, y, z, u[0], u[1], u[2], t, maxb, ph);
}

typedef struct ka_job {
    const cl_box* box; const cl_optical_params* op; const cl_readout* ro;
    const cl_time_binning* tb;
    /* point mode */
    const float *px, *py, *pz, *pt; int32_t npos;
    /* segment mode */
    const int64_t* offs; int64_t nsrc;
    uint64_t seed, pid0; float tau; int32_t maxb;
    int64_t k0, k1;
    uint8_t* status; int16_t* idx; float* t; int32_t* bounces; int32_t* nscat;
    int64_t steps;
} ka_job;

static void* ka_worker(void* arg)
{
    ka_job* j = (ka_job*)arg;
    int64_t steps = 0;
    int64_t src = 0;
    if (j->offs) {  /* first source containing k0 */
        int64_t lo = 0, hi = j->nsrc - 1;
        while (lo < hi) {
            int64_t mid = (lo + hi + 1) / 2;
            if (j->offs[mid] <= j->k0) lo = mid; else hi = mid - 1;
        }
        src = lo;
    }
    for (int64_t k = j->k0; k < j->k1; ++k) {
        int64_t p;
        if (j->offs) {
            while (j->offs[src + 1] <= k) ++src;
            p = src;
        } else {
            p = k % j->npos;
        }
        or_photon ph;
        ka_photon(j->box, j->op, j->ro, j->tb, j->seed, j->pid0 + (uint64_t)k + 1u,
                  j->px[p], j->py[p], j->pz[p], j->pt ? j->pt[p] : 0.0f,
                  j->tau, j->maxb, &ph);
        j->status[k] = (uint8_t)ph.status;
        j->idx[k] = ph.idx;
        j->t[k] = ph.t;
        j->bounces[k] = ph.bounces;
        j->nscat[k] = ph.nscat;
        steps += ph.steps;
    }
    j->steps = steps;
    return NULL;
}

static int run_records(ka_job* proto, int64_t n, int nthreads, int64_t* steps)
{
    int nt = clamp_threads(nthreads, n);
    ka_job* jobs = (ka_job*)calloc((size_t)nt, sizeof(ka_job));
    pthread_t* th = (pthread_t*)calloc((size_t)nt, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1; }
    for (int t = 0; t < nt; ++t) {
        jobs[t] = *proto;
        jobs[t].k0 = n * t / nt;
        jobs[t].k1 = n * (t + 1) / nt;
    }
    for (int t = 1; t < nt; ++t) pthread_create(&th[t], NULL, ka_worker, &jobs[t]);
    ka_worker(&jobs[0]);
    for (int t = 1; t < nt; ++t) pthread_join(th[t], NULL);
    int64_t s = 0;
    for (int t = 0; t < nt; ++t) s += jobs[t].steps;
    if (steps) *steps = s;
    free(jobs); free(th);
    return 0;
}

typedef struct rec_buf {
    uint8_t* status; int16_t* idx; float* t; int32_t* bounces; int32_t* nscat;
} rec_buf;

static int rec_alloc(rec_buf* r, int64_t n)
{
    size_t m = n > 0 ? (size_t)n : 1;
    r->status = (uint8_t*)malloc(m);
    r->idx = (int16_t*)malloc(m * sizeof(int16_t));
    r->t = (float*)malloc(m * sizeof(float));
    r->bounces = (int32_t*)malloc(m * sizeof(int32_t));
    r->nscat = (int32_t*)malloc(m * sizeof(int32_t));
    return (r->status && r->idx && r->t && r->bounces && r->nscat) ? 0 : -1;
}

static void rec_free(rec_buf* r)
{
    free(r->status); free(r->idx); free(r->t); free(r->bounces); free(r->nscat);
}

static void rec_export(const rec_buf* r, int64_t n, const cl_records* out)
{
    if (!out) return;
    if (out->status) memcpy(out->status, r->status, (size_t)n);
    if (out->idx) memcpy(out->idx, r->idx, (size_t)n * sizeof(int16_t));
    if (out->t) memcpy(out->t, r->t, (size_t)n * sizeof(float));
    if (out->bounces) memcpy(out->bounces, r->bounces, (size_t)n * sizeof(int32_t));
}

int or_run_photons_ka(const cl_box* box, const cl_optical_params* op,
                      const cl_readout* ro, const cl_time_binning* tb,
                      const float* px, const float* py, const float* pz,
                      const float* pt, int32_t npos,
                      int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                      float tau_ns, int32_t max_bounces, int nthreads,
                      uint32_t* counts, float* first_ns, cl_counters* counters,
                      const cl_records* records, int64_t* steps)
{
    if (npos < 1 || n_photons < 0) return -1;
    rec_buf r;
    if (rec_alloc(&r, n_photons)) { rec_free(&r); return -1; }
    ka_job proto;
    memset(&proto, 0, sizeof proto);
    proto.box = box; proto.op = op; proto.ro = ro; proto.tb = tb;
    proto.px = px; proto.py = py; proto.pz = pz; proto.pt = pt; proto.npos = npos;
    proto.seed = seed; proto.pid0 = pid_offset; proto.tau = tau_ns; proto.maxb = max_bounces;
    proto.status = r.status; proto.idx = r.idx; proto.t = r.t;
    proto.bounces = r.bounces; proto.nscat = r.nscat;
    if (run_records(&proto, n_photons, nthreads, steps)) { rec_free(&r); return -1; }

    if (counts && first_ns && counters) {
        /* host reduction, src/kernel.jl:337-365 (plus nscat, which the
         * reference's CPU path counts in Accumulator.nscat) */
        const int32_t nx = ro->grid.nx, ny = ro->grid.ny;
        size_t ncell = (size_t)nx * ny;
        memset(counts, 0, ncell * (size_t)(tb->nbins + 1) * sizeof(uint32_t));
        for (size_t i = 0; i < ncell; ++i) first_ns[i] = INFINITY;
        cl_counters c;
        memset(&c, 0, sizeof c);
        for (int64_t k = 0; k < n_photons; ++k) {
            int32_t s = r.status[k];
            c.nscat += r.nscat[k];
            if (s == CL_STATUS_DETECTED) {
                int32_t lin = r.idx[k];
                if (lin < 0) { c.ndet_front += 1; lin = -lin; }
                int32_t ii = (lin - 1) % nx + 1;
                int32_t jj = (lin - 1) / nx + 1;
                float t = r.t[k];
                int32_t bin = time_bin(tb, t);
                size_t cell = (size_t)(ii - 1) + (size_t)nx * (size_t)(jj - 1);
                counts[cell + ncell * (size_t)(bin - 1)] += 1u;
                if (t < first_ns[cell]) first_ns[cell] = t;
                c.ndet += 1;
                c.sum_bounces_det += r.bounces[k];
            } else if (s == CL_STATUS_ABS_BULK) c.nabs_bulk += 1;
            else if (s == CL_STATUS_ABS_WALL) c.nabs_wall += 1;
            else if (s == CL_STATUS_ABS_SIPM) c.nabs_sipm += 1;
            else if (s == CL_STATUS_ABS_SUR) c.nabs_sur += 1;
            else c.ncap += 1;
        }
        *counters = c;
    }
    rec_export(&r, n_photons, records);
    rec_free(&r);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Segments: the per-event reduction of flush!, src/events.jl:65-91           */
/* ------------------------------------------------------------------------ */
int or_run_segments(const cl_box* box, const cl_optical_params* op,
                    const cl_readout* ro, const cl_time_binning* tb,
                    const float* sx, const float* sy, const float* sz,
                    const float* st, const int64_t* src_offsets,
                    const int32_t* src_segment, int64_t n_src, int64_t n_segments,
                    uint64_t seed, uint64_t pid_offset, float tau_ns,
                    int32_t max_bounces, int nthreads,
                    uint32_t* maps, float* tmin, int32_t* npe,
                    cl_counters* counters, const cl_records* records,
                    int64_t* steps)
{
    if (n_src < 1 || n_segments < 1 || src_offsets[0] != 0) return -1;
    int64_t n = src_offsets[n_src];
    rec_buf r;
    if (rec_alloc(&r, n)) { rec_free(&r); return -1; }
    ka_job proto;
    memset(&proto, 0, sizeof proto);
    proto.box = box; proto.op = op; proto.ro = ro; proto.tb = tb;
    proto.px = sx; proto.py = sy; proto.pz = sz; proto.pt = st; proto.npos = 1;
    proto.offs = src_offsets; proto.nsrc = n_src;
    proto.seed = seed; proto.pid0 = pid_offset; proto.tau = tau_ns; proto.maxb = max_bounces;
    proto.status = r.status; proto.idx = r.idx; proto.t = r.t;
    proto.bounces = r.bounces; proto.nscat = r.nscat;
    if (run_records(&proto, n, nthreads, steps)) { rec_free(&r); return -1; }

    const int32_t nx = ro->grid.nx, ny = ro->grid.ny;
    const size_t ncell = (size_t)nx * ny;
    memset(maps, 0, ncell * (size_t)n_segments * sizeof(uint32_t));
    for (size_t i = 0; i < ncell * (size_t)n_segments; ++i) tmin[i] = INFINITY;
    memset(npe, 0, (size_t)n_segments * sizeof(int32_t));
    cl_counters c;
    memset(&c, 0, sizeof c);
    for (int64_t s = 0; s < n_src; ++s) {
        int64_t seg = src_segment[s];
        for (int64_t k = src_offsets[s]; k < src_offsets[s + 1]; ++k) {
            int32_t stt = r.status[k];
            c.nscat += r.nscat[k];
            if (stt == CL_STATUS_DETECTED) {
                int32_t lin = r.idx[k];
                if (lin < 0) { c.ndet_front += 1; lin = -lin; }
                int32_t ii = (lin - 1) % nx + 1;
                int32_t jj = (lin - 1) / nx + 1;
                size_t cell = (size_t)(ii - 1) + (size_t)nx * (size_t)(jj - 1) + ncell * (size_t)seg;
                maps[cell] += 1u;
                if (r.t[k] < tmin[cell]) tmin[cell] = r.t[k];
                npe[seg] += 1;
                c.ndet += 1;
                c.sum_bounces_det += r.bounces[k];
            } else if (stt == CL_STATUS_ABS_BULK) c.nabs_bulk += 1;
            else if (stt == CL_STATUS_ABS_WALL) c.nabs_wall += 1;
            else if (stt == CL_STATUS_ABS_SIPM) c.nabs_sipm += 1;
            else if (stt == CL_STATUS_ABS_SUR) c.nabs_sur += 1;
            else c.ncap += 1;
        }
    }
    *counters = c;
    rec_export(&r, n, records);
    rec_free(&r);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Batch helpers for tests                                                   */
/* ------------------------------------------------------------------------ */
void or_eval_batch(int fn, const float* in, float* out, int64_t n)
{
    for (int64_t i = 0; i < n; ++i) {
        float x = in[i];
        out[i] = fn == 0 ? or_logf(x) : (fn == 1 ? or_sinf(x) : or_cosf(x));
    }
}

void or_randu_batch(uint64_t seed, int64_t n_streams, int32_t n_per, float* out)
{
    for (int64_t k = 0; k < n_streams; ++k) {
        or_stream s;
        or_stream_init(&s, seed, (uint64_t)k + 1u);
        for (int32_t i = 0; i < n_per; ++i) out[k * n_per + i] = or_randu(&s);
    }
}

void or_philox_batch(const uint32_t* ctr, uint64_t seed, int64_t n, uint32_t* out)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int64_t k = 0; k < n; ++k) or_philox4x32(ctr + 4 * k, key, out + 4 * k);
}
