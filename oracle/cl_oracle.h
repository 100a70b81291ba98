/*
 * cl_oracle.h — CPU restatement of CryspLight's optical-photon transport.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against (and the timed CPU baseline); the product never links or calls it.
 *
 * It restates, draw for draw and operation for operation, the reference's
 * Julia code: src/philox.jl, src/geometry.jl, src/optics.jl,
 * src/generation.jl, src/transport.jl, the record path of src/kernel.jl and
 * the per-event reduction of src/events.jl.  Parameter structs come from the
 * public header so tests can pass the same values to both sides.
 *
 * Elementary functions: Julia Base evaluates Float32 log/sin/cos itself (not
 * in the reference tree).  The oracle evaluates them in Float64 with the C
 * library and rounds once to Float32, i.e. the correctly rounded value except
 * in vanishingly rare near-halfway cases.  Whether Julia returns exactly these
 * bits is not pinned here (no Julia in this environment): see the oracle's
 * section of the design notes.
 */
#ifndef CL_ORACLE_H
#define CL_ORACLE_H

#include <stdint.h>
#include "../include/crysplight_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Philox4x32-10, src/philox.jl:5-62 ---- */
void or_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

typedef struct or_stream {
    uint32_t key[2];
    uint32_t id_lo, id_hi;
    uint32_t block;
    uint32_t buf[4];
    int      i;
} or_stream;

void     or_stream_init(or_stream* s, uint64_t seed, uint64_t photon_id);
uint32_t or_next_u32(or_stream* s);
float    or_randu(or_stream* s);

/* ---- elementary functions (Float64 evaluation, one rounding) ---- */
float or_logf(float x);
float or_sinf(float x);
float or_cosf(float x);

/* ---- geometry / optics / generation ---- */
int32_t or_wall_hit(float x, float y, float z, float ux, float uy, float uz,
                    const cl_box* box, float* d);
int     or_fresnel(float n1, float n2, float cosi, float* R);   /* returns tir */
void    or_isotropic_dir(or_stream* s, float u[3]);
float   or_emission_time(or_stream* s, float tau_ns);
float   or_gaussian(or_stream* s);
void    or_lambertian_dir(or_stream* s, int32_t face, float u[3]);
void    or_rayleigh_dir(or_stream* s, const float u[3], float v[3]);
/* returns transmitted; v = outgoing direction (unchanged when transmitted) */
int     or_surface_interact(or_stream* s, const float u[3], int32_t face,
                            float n_crystal, float sigma_alpha, float v[3]);

/* ---- Accumulator, src/transport.jl:64-108 ---- */
typedef struct or_acc {
    uint32_t*   counts;     /* nx*ny*(nbins+1), column-major */
    float*      first_ns;   /* nx*ny */
    cl_counters c;
    int32_t     nx, ny, nbins;
} or_acc;

/* Per-photon outcome (the kernel twin's record plus diagnostics). */
typedef struct or_photon {
    int32_t status;
    int16_t idx;
    float   t;
    int32_t bounces;
    int32_t nscat;
    int32_t steps;
} or_photon;

/* propagate_photon!, src/transport.jl:118-234.  acc may be NULL. */
int32_t or_propagate_photon(or_acc* acc, const cl_box* box,
                            const cl_optical_params* op, const cl_readout* ro,
                            const cl_time_binning* tb, or_stream* s,
                            float x, float y, float z,
                            float ux, float uy, float uz, float t0,
                            int32_t max_bounces, or_photon* out);

/* run_photons!, src/transport.jl:245-273: nthreads static-striped threads,
 * pid = 1..n, source plist[(pid-1) % npos], t0 = emission time only.
 * counts/first_ns are overwritten. */
int or_run_photons(const cl_box* box, const cl_optical_params* op,
                   const cl_readout* ro, const cl_time_binning* tb,
                   const float* px, const float* py, const float* pz, int32_t npos,
                   int64_t n_photons, uint64_t seed, float tau_ns,
                   int32_t max_bounces, int nthreads,
                   uint32_t* counts, float* first_ns, cl_counters* counters);

/* transport_kernel! + run_photons_ka!'s host reduction, src/kernel.jl:159-367:
 * pid = pid_offset + k + 1, source k % npos, t0 = pt[j] + emission time.
 * records (any field may be NULL) are indexed by k.  counts/first_ns/counters
 * may be NULL to skip the reduction.  Also returns total steps if steps!=NULL. */
int or_run_photons_ka(const cl_box* box, const cl_optical_params* op,
                      const cl_readout* ro, const cl_time_binning* tb,
                      const float* px, const float* py, const float* pz,
                      const float* pt, int32_t npos,
                      int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                      float tau_ns, int32_t max_bounces, int nthreads,
                      uint32_t* counts, float* first_ns, cl_counters* counters,
                      const cl_records* records, int64_t* steps);

/* Segmented transport (sources with photon counts grouped into segments):
 * the per-event reduction of src/events.jl:65-91 over records, generalised to
 * any source/segment layout.  Outputs as cl_run_segments. */
int or_run_segments(const cl_box* box, const cl_optical_params* op,
                    const cl_readout* ro, const cl_time_binning* tb,
                    const float* sx, const float* sy, const float* sz,
                    const float* st, const int64_t* src_offsets,
                    const int32_t* src_segment, int64_t n_src, int64_t n_segments,
                    uint64_t seed, uint64_t pid_offset, float tau_ns,
                    int32_t max_bounces, int nthreads,
                    uint32_t* maps, float* tmin, int32_t* npe,
                    cl_counters* counters, const cl_records* records,
                    int64_t* steps);

/* Reference-operation counter (analysis build with -DOR_COUNT_OPS only). */
uint64_t or_ops_read(void);
void or_ops_reset(void);

/* Batch helpers for tests. */
void or_eval_batch(int fn, const float* in, float* out, int64_t n);
void or_randu_batch(uint64_t seed, int64_t n_streams, int32_t n_per, float* out);
void or_philox_batch(const uint32_t* ctr, uint64_t seed, int64_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif
