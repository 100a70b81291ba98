// cl_gamma.cpp — host-side 511 keV gamma stage of the event pipeline.
//
// Restates the reference's vendored gamma core (src/gamma/*.jl: XCOM log-log
// cross sections, exponential free path, Compton / photoelectric / pair
// choice, Klein-Nishina sampling by Butcher-Messel, 10 keV cut, slab exit of
// an origin-centred box), its crystal-frame bridge (src/gamma_interface.jl:
// cm/MeV -> mm/keV, deposit time = path / c, process codes) and the photon
// count per deposit (rand_poisson, src/events.jl:11-22), for the per-event
// loop of run_events! (src/events.jl:93-118).
//
// Random numbers: the reference draws from Julia's Xoshiro seeded by
// hash((seed, ev)), which cannot be reproduced outside Julia.  Each event here
// draws from its own Philox4x32-10 stream (key = seed, counter = (event lo,
// event hi, block, 0x67616d6d)), in the reference's order; Float64 uniforms
// are 53-bit, [0, 1).  Standard normals for the Poisson Gaussian branch come
// from Box-Muller.  Results are therefore statistically, not bitwise,
// equivalent to the reference's event pipeline.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "../../include/crysplight_cuda.h"

namespace {

constexpr double ME = 0.51099895;          // electron rest mass [MeV], src/gamma/sampling.jl:3
constexpr double C_CM_NS = 29.9792458;     // src/gamma_interface.jl:7
constexpr double EGAMMA_CUT = 0.010;       // src/gamma/gtransport.jl:44
constexpr double SURFACE_EPS = 1e-10;      // src/gamma/ggeometry.jl:6
constexpr double PARALLEL_EPS = 1e-20;
constexpr double TWO_PI = 6.283185307179586;

thread_local char g_err[256];

// ---- Philox stream of Float64 uniforms ----
struct GammaRng {
    uint32_t k0, k1, ev_lo, ev_hi, block;
    uint32_t buf[4];
    int n;
    bool have_spare;
    double spare;
};

inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[1] = (uint32_t)p1;
        c[3] = (uint32_t)p0;
        c[0] = n0;
        c[2] = n2;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

inline void rng_init(GammaRng& g, uint64_t seed, uint64_t ev)
{
    g.k0 = (uint32_t)seed; g.k1 = (uint32_t)(seed >> 32);
    g.ev_lo = (uint32_t)ev; g.ev_hi = (uint32_t)(ev >> 32);
    g.block = 0; g.n = 0; g.have_spare = false; g.spare = 0.0;
}

inline uint32_t rng_u32(GammaRng& g)
{
    if (g.n == 0) {
        g.buf[0] = g.ev_lo; g.buf[1] = g.ev_hi; g.buf[2] = g.block++; g.buf[3] = 0x67616d6du;
        philox(g.buf, g.k0, g.k1);
        g.n = 4;
    }
    return g.buf[4 - g.n--];
}

// rand(rng): uniform in [0, 1) with 53 random bits.
inline double rand01(GammaRng& g)
{
    const uint64_t hi = rng_u32(g), lo = rng_u32(g);
    return (double)(((hi << 32) | lo) >> 11) * 0x1p-53;
}

// randn(rng) by Box-Muller (two uniforms per pair of normals).
inline double randn(GammaRng& g)
{
    if (g.have_spare) { g.have_spare = false; return g.spare; }
    double u1;
    do { u1 = rand01(g); } while (u1 <= 0.0);
    const double u2 = rand01(g);
    const double r = std::sqrt(-2.0 * std::log(u1));
    g.spare = r * std::sin(TWO_PI * u2);
    g.have_spare = true;
    return r * std::cos(TWO_PI * u2);
}

}  // namespace

// ---- material: XCOM tables, src/gamma/gmaterials.jl + nist_data.jl ----
struct cl_gamma_material {
    double density;
    std::vector<double> E, logE, incoh, photo, pair, log_incoh, log_photo, log_pair;
};

namespace {

std::vector<double> prelog(const std::vector<double>& v)
{
    std::vector<double> o(v.size());
    for (size_t i = 0; i < v.size(); ++i) o[i] = v[i] > 0.0 ? std::log(v[i]) : -INFINITY;
    return o;
}

// interp_loglog_prelogged, src/gamma/nist_data.jl
inline double interp(double lx, const std::vector<double>& log_xp, const std::vector<double>& log_fp,
                     const std::vector<double>& fp, size_t lo)
{
    const size_t hi = lo + 1;
    const double fl = fp[lo], fh = fp[hi];
    if (fl <= 0.0) return 0.0;
    if (fh <= 0.0) return fl;
    const double t = (lx - log_xp[lo]) / (log_xp[hi] - log_xp[lo]);
    return std::exp(log_fp[lo] + t * (log_fp[hi] - log_fp[lo]));
}

// sigma_macro, src/gamma/gmaterials.jl:45-57: (Sigma_C, Sigma_Ph, Sigma_P) [1/cm]
inline void sigma_macro(const cl_gamma_material* m, double E, double out[3])
{
    const size_t n = m->E.size();
    if (n == 0) { out[0] = out[1] = out[2] = 0.0; return; }
    const double lx = std::log(E);
    // searchsortedlast(E, x) (1-based) clamped to [1, n-1] -> 0-based [0, n-2]
    size_t k = (size_t)(std::upper_bound(m->E.begin(), m->E.end(), E) - m->E.begin());  // count <= E
    size_t lo = k == 0 ? 0 : k - 1;
    if (lo > n - 2) lo = n - 2;
    out[0] = interp(lx, m->logE, m->log_incoh, m->incoh, lo) * m->density;
    out[1] = interp(lx, m->logE, m->log_photo, m->photo, lo) * m->density;
    out[2] = interp(lx, m->logE, m->log_pair, m->pair, lo) * m->density;
}

// distance_to_exit for an origin-centred box (half-extents h), src/gamma/ggeometry.jl:13-38
inline double distance_to_exit(const double p[3], const double d[3], const double h[3])
{
    double t_near = -INFINITY, t_far = INFINITY;
    for (int i = 0; i < 3; ++i) {
        if (std::fabs(d[i]) > PARALLEL_EPS) {
            const double t1 = (-h[i] - p[i]) / d[i], t2 = (h[i] - p[i]) / d[i];
            t_near = std::max(t_near, std::min(t1, t2));
            t_far = std::min(t_far, std::max(t1, t2));
        } else if (p[i] < -h[i] || p[i] > h[i]) {
            return INFINITY;
        }
    }
    if (t_far < t_near) return INFINITY;
    return t_far > SURFACE_EPS ? t_far : INFINITY;
}

// sample_compton (Butcher-Messel), src/gamma/sampling.jl:28-40
inline void sample_compton(double E, GammaRng& g, double* Eprime, double* cost)
{
    const double eps0 = ME / (ME + 2.0 * E);
    const double a1 = -std::log(eps0);
    const double a2 = (1.0 - eps0 * eps0) / 2.0;
    for (;;) {
        const double r1 = rand01(g), r2 = rand01(g), r3 = rand01(g);
        const double eps = r1 < a1 / (a1 + a2) ? std::pow(eps0, r2)
                                               : std::sqrt(eps0 * eps0 + (1.0 - eps0 * eps0) * r2);
        const double omc = (1.0 - eps) * ME / (E * eps);
        const double sin2 = std::min(1.0, std::max(0.0, omc * (2.0 - omc)));
        const double gg = 1.0 - eps * sin2 / (1.0 + eps * eps);
        if (gg >= r3) { *Eprime = eps * E; *cost = 1.0 - omc; return; }
    }
}

// rotate_to_global, src/gamma/sampling.jl:48-64
inline void rotate_to_global(const double l[3], const double ref[3], double out[3])
{
    const double n = std::sqrt(ref[0] * ref[0] + ref[1] * ref[1] + ref[2] * ref[2]);
    const double rx = ref[0] / n, ry = ref[1] / n, rz = ref[2] / n;
    if (std::fabs(rz) > 0.99999) {
        const double s = rz > 0.0 ? 1.0 : (rz < 0.0 ? -1.0 : 0.0);
        out[0] = l[0] * s; out[1] = l[1] * s; out[2] = l[2] * s;
        return;
    }
    const double rp = std::sqrt(rx * rx + ry * ry);
    const double e1x = -rz * rx / rp, e1y = -rz * ry / rp, e1z = -(rz * rz - 1.0) / rp;
    const double e2x = -ry / rp, e2y = rx / rp;
    out[0] = l[0] * e1x + l[1] * e2x + l[2] * rx;
    out[1] = l[0] * e1y + l[1] * e2y + l[2] * ry;
    out[2] = l[0] * e1z + l[2] * rz;
}

struct Deposit { float x, y, z, e_kev, t_ns; int32_t proc; };   // proc: 0 photo, 1 compton, 2 below cut

// propagate_photon (src/gamma/gtransport.jl:44-81) + gamma_deposits
// (src/gamma_interface.jl:30-49): deposits in the crystal frame.
void gamma_deposits(const cl_gamma_material* m, const cl_box* box, const float entry[3],
                    const double dir0[3], double e0, GammaRng& g, std::vector<Deposit>& out)
{
    out.clear();
    const double h[3] = {box->L[0] / 20.0, box->L[1] / 20.0, box->L[2] / 20.0};   // half-extents, cm
    // p0 = ((entry - L/2)/10) is Float32 arithmetic in the reference, then Float64
    double pos[3] = {(double)((entry[0] - box->L[0] / 2.0f) / 10.0f),
                     (double)((entry[1] - box->L[1] / 2.0f) / 10.0f),
                     (double)((entry[2] - box->L[2] / 2.0f) / 10.0f)};
    double dir[3] = {dir0[0], dir0[1], dir0[2]};
    const double dn = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    dir[0] /= dn; dir[1] /= dn; dir[2] /= dn;
    double prev[3] = {pos[0], pos[1], pos[2]};
    double path = 0.0, E = e0;
    auto record = [&](const double p[3], double e_dep, int proc) {
        path += std::sqrt((p[0] - prev[0]) * (p[0] - prev[0]) + (p[1] - prev[1]) * (p[1] - prev[1]) +
                          (p[2] - prev[2]) * (p[2] - prev[2]));
        prev[0] = p[0]; prev[1] = p[1]; prev[2] = p[2];
        if (e_dep > 0.0)
            out.push_back({(float)(p[0] * 10 + box->L[0] / 2.0f), (float)(p[1] * 10 + box->L[1] / 2.0f),
                           (float)(p[2] * 10 + box->L[2] / 2.0f), (float)(e_dep * 1000),
                           (float)(path / C_CM_NS), proc});
    };
    for (int guard = 0; guard < 100000; ++guard) {
        double S[3];
        sigma_macro(m, E, S);
        const double Sig = S[0] + S[1] + S[2];
        const double s = Sig > 0.0 ? -std::log(rand01(g)) / Sig : INFINITY;
        const double d_exit = distance_to_exit(pos, dir, h);
        if (s >= d_exit) {                       // escape record (no deposit)
            const double p[3] = {pos[0] + d_exit * dir[0], pos[1] + d_exit * dir[1], pos[2] + d_exit * dir[2]};
            record(p, 0.0, -1);
            return;
        }
        pos[0] += s * dir[0]; pos[1] += s * dir[1]; pos[2] += s * dir[2];
        // sample_process / sample_interaction, src/gamma/sampling.jl:10-26, 85-98
        const double r = rand01(g);
        const double PC = S[0] / Sig, PP = S[2] / Sig;
        if (r < PC) {
            double Ep, cost;
            sample_compton(E, g, &Ep, &cost);
            const double phi = TWO_PI * rand01(g);
            const double sint = std::sqrt(std::max(0.0, 1.0 - cost * cost));
            const double l[3] = {sint * std::cos(phi), sint * std::sin(phi), cost};
            double nd[3];
            rotate_to_global(l, dir, nd);
            record(pos, E - Ep, 1);
            dir[0] = nd[0]; dir[1] = nd[1]; dir[2] = nd[2];
            E = Ep;
            if (E < EGAMMA_CUT) { record(pos, E, 2); return; }
        } else {
            (void)PP;                            // pair (closed below 1.022 MeV) and photoelectric:
            record(pos, E, 0);                   // full absorption, history ends
            return;
        }
    }
}

// rand_poisson, src/events.jl:11-22
int64_t rand_poisson(GammaRng& g, double lam)
{
    if (lam <= 0.0) return 0;
    if (lam > 50.0) {
        const double v = std::nearbyint(lam + std::sqrt(lam) * randn(g));   // round: ties to even
        return v > 0.0 ? (int64_t)v : 0;
    }
    const double L = std::exp(-lam);
    int64_t k = 0;
    double p = 1.0;
    for (;;) {
        p *= rand01(g);
        if (p < L) return k;
        k += 1;
    }
}

struct EventOut {
    float edep, xyz1[3], e1, xyz2[3], e2, er;
    int8_t int_type;
    int16_t n_int;
};

// One event of run_events! (src/events.jl:93-118): entry point, deposits,
// truth, photons per deposit.
void one_event(const cl_gamma_material* m, const cl_box* box, uint64_t seed, uint64_t ev,
               double e0_mev, double yield, EventOut& eo, std::vector<Deposit>& deps,
               std::vector<int64_t>& nph)
{
    GammaRng g;
    rng_init(g, seed, ev);
    const float e0_kev = (float)(e0_mev * 1000);
    memset(&eo, 0, sizeof eo);
    eo.er = e0_kev;
    eo.int_type = -1;
    const float entry[3] = {(float)(rand01(g) * box->L[0]), (float)(rand01(g) * box->L[1]), 0.0f};
    const double dir[3] = {0.0, 0.0, 1.0};
    gamma_deposits(m, box, entry, dir, e0_mev, g, deps);
    nph.clear();
    if (deps.empty()) return;
    int ncompt = 0;
    for (const Deposit& d : deps) ncompt += d.proc == 1;
    eo.int_type = (int8_t)std::min(ncompt, 127);
    eo.n_int = (int16_t)std::min<size_t>(deps.size(), 32767);
    eo.xyz1[0] = deps[0].x; eo.xyz1[1] = deps[0].y; eo.xyz1[2] = deps[0].z;
    eo.e1 = deps[0].e_kev;
    if (deps.size() >= 2) {
        eo.xyz2[0] = deps[1].x; eo.xyz2[1] = deps[1].y; eo.xyz2[2] = deps[1].z;
        eo.e2 = deps[1].e_kev;
    }
    eo.er = e0_kev - eo.e1 - eo.e2;
    for (const Deposit& d : deps) {
        eo.edep += d.e_kev;
        nph.push_back(rand_poisson(g, yield * (double)d.e_kev / 1000));
    }
}

}  // namespace

extern "C" {

int cl_gamma_material_create(cl_gamma_material** out, const double* E_MeV, const double* incoherent,
                             const double* photoelectric, const double* pair_nuclear,
                             const double* pair_electron, int32_t n, double density)
{
    g_err[0] = 0;
    if (!out || n < 0 || (n > 0 && (!E_MeV || !incoherent || !photoelectric || !pair_nuclear || !pair_electron))) {
        snprintf(g_err, sizeof g_err, "cl_gamma_material_create: bad arguments");
        return CL_ERR_ARG;
    }
    if (n == 1) {
        snprintf(g_err, sizeof g_err, "cl_gamma_material_create: need at least 2 energies");
        return CL_ERR_ARG;
    }
    cl_gamma_material* m = new (std::nothrow) cl_gamma_material();
    if (!m) return CL_ERR_OOM;
    m->density = density;
    // _prepare_xcom_energy: nudge duplicate K-edge energies apart, src/gamma/gmaterials.jl
    m->E.assign(E_MeV, E_MeV + n);
    for (int32_t i = 1; i < n; ++i)
        if (m->E[i] <= m->E[i - 1]) m->E[i] = m->E[i - 1] * (1.0 + 1e-9);
    m->logE.resize(n);
    for (int32_t i = 0; i < n; ++i) m->logE[i] = std::log(m->E[i]);
    m->incoh.assign(incoherent, incoherent + n);
    m->photo.assign(photoelectric, photoelectric + n);
    m->pair.resize(n);
    for (int32_t i = 0; i < n; ++i) m->pair[i] = pair_nuclear[i] + pair_electron[i];
    m->log_incoh = prelog(m->incoh);
    m->log_photo = prelog(m->photo);
    m->log_pair = prelog(m->pair);
    *out = m;
    return CL_OK;
}

void cl_gamma_material_destroy(cl_gamma_material* m) { delete m; }

const char* cl_gamma_last_error(void) { return g_err; }

int cl_gamma_sigma(const cl_gamma_material* m, double E_MeV, double* sigma3)
{
    if (!m || !sigma3) return CL_ERR_ARG;
    sigma_macro(m, E_MeV, sigma3);
    return CL_OK;
}

int cl_gamma_deposits(const cl_gamma_material* m, const cl_box* box, const float* entry_mm,
                      const double* dir, double e0_mev, uint64_t seed, uint64_t stream,
                      float* dep6, int32_t max_dep, int32_t* n_dep)
{
    if (!m || !box || !entry_mm || !dir || !dep6 || !n_dep || max_dep < 0) return CL_ERR_ARG;
    GammaRng g;
    rng_init(g, seed, stream);
    std::vector<Deposit> deps;
    gamma_deposits(m, box, entry_mm, dir, e0_mev, g, deps);
    *n_dep = (int32_t)deps.size();
    if ((int32_t)deps.size() > max_dep) {
        snprintf(g_err, sizeof g_err, "cl_gamma_deposits: %zu deposits exceed capacity %d", deps.size(), (int)max_dep);
        return CL_ERR_ARG;
    }
    for (size_t i = 0; i < deps.size(); ++i) {
        float* o = dep6 + 6 * i;
        o[0] = deps[i].x; o[1] = deps[i].y; o[2] = deps[i].z;
        o[3] = deps[i].e_kev; o[4] = deps[i].t_ns; o[5] = (float)deps[i].proc;
    }
    return CL_OK;
}

int64_t cl_rand_poisson(uint64_t seed, uint64_t stream, double lam)
{
    GammaRng g;
    rng_init(g, seed, stream);
    return rand_poisson(g, lam);
}

int cl_gamma_events(const cl_gamma_material* m, const cl_box* box, int64_t ev0, int64_t n_events,
                    uint64_t seed, double e0_mev, double yield_per_mev, int nthreads,
                    float* edep, float* xyz1, float* e1, float* xyz2, float* e2, float* er,
                    int8_t* int_type, int16_t* n_int,
                    int64_t max_deposits, float* dep_xyz, float* dep_t, int32_t* dep_event,
                    int64_t* dep_photons, int64_t* n_deposits)
{
    g_err[0] = 0;
    if (!m || !box || n_events < 0 || ev0 < 0 || !edep || !xyz1 || !e1 || !xyz2 || !e2 || !er ||
        !int_type || !n_int || !n_deposits || max_deposits < 0 ||
        (max_deposits > 0 && (!dep_xyz || !dep_t || !dep_event || !dep_photons))) {
        snprintf(g_err, sizeof g_err, "cl_gamma_events: bad arguments");
        return CL_ERR_ARG;
    }
    if (nthreads < 1) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    if ((int64_t)nthreads > n_events) nthreads = (int)std::max<int64_t>(1, n_events);
    // phase 1: events in parallel (deterministic per event), per-thread deposit lists
    struct Part { std::vector<Deposit> deps; std::vector<int64_t> nph; std::vector<int32_t> evi; };
    std::vector<Part> parts((size_t)nthreads);
    auto work = [&](int t) {
        Part& P = parts[(size_t)t];
        std::vector<Deposit> d;
        std::vector<int64_t> nph;
        const int64_t a = n_events * t / nthreads, b = n_events * (t + 1) / nthreads;
        for (int64_t i = a; i < b; ++i) {
            EventOut eo;
            one_event(m, box, seed, (uint64_t)(ev0 + i + 1), e0_mev, yield_per_mev, eo, d, nph);
            edep[i] = eo.edep; e1[i] = eo.e1; e2[i] = eo.e2; er[i] = eo.er;
            for (int c = 0; c < 3; ++c) { xyz1[3 * i + c] = eo.xyz1[c]; xyz2[3 * i + c] = eo.xyz2[c]; }
            int_type[i] = eo.int_type;
            n_int[i] = eo.n_int;
            for (size_t k = 0; k < d.size(); ++k) {
                P.deps.push_back(d[k]);
                P.nph.push_back(nph[k]);
                P.evi.push_back((int32_t)i);
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    // phase 2: concatenate in event order (threads own contiguous event ranges)
    int64_t total = 0;
    for (const Part& P : parts) total += (int64_t)P.deps.size();
    *n_deposits = total;
    if (total > max_deposits) {
        snprintf(g_err, sizeof g_err, "cl_gamma_events: %lld deposits exceed capacity %lld",
                 (long long)total, (long long)max_deposits);
        return CL_ERR_ARG;
    }
    int64_t o = 0;
    for (const Part& P : parts) {
        for (size_t k = 0; k < P.deps.size(); ++k, ++o) {
            dep_xyz[3 * o] = P.deps[k].x; dep_xyz[3 * o + 1] = P.deps[k].y; dep_xyz[3 * o + 2] = P.deps[k].z;
            dep_t[o] = P.deps[k].t_ns;
            dep_event[o] = P.evi[k];
            dep_photons[o] = P.nph[k];
        }
    }
    return CL_OK;
}

}  // extern "C"
