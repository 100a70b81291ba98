/*
 * crysplight_cuda.h — C-ABI of the B200 optical-photon transport engine.
 *
 * Drop-in boundary for CryspLight's transport call.  The reference has no FFI:
 * its seam is the Julia function
 *
 *   run_photons_ka!(box, op, ro, tb; n_photons, seed, pos | positions, t0s,
 *                   pid_offset, tau_ns, max_bounces, ArrayT, return_records)
 *       -> Accumulator [, records]                      (src/kernel.jl:312-367)
 *
 * and its CPU twin run_photons! (src/transport.jl:245-273).  The entry points
 * below take the same arguments as plain pointers and sizes, so a Julia
 * `ccall` (or ctypes, or C) binds them directly.  The parameter structs are
 * layout-identical to the Julia isbits structs (C rules, Bool = uint8_t), so a
 * Julia `Ref(op)` can be passed where a `const cl_optical_params*` is expected.
 *
 * Conventions (kept from the reference):
 *   - photon ids are 1-based: the k-th photon of a call (k = 0..n-1) draws
 *     from the Philox4x32-10 stream key = (seed lo, seed hi),
 *     counter = (pid lo, pid hi, block, 0) with pid = pid_offset + k + 1
 *     (src/philox.jl:30-48, src/kernel.jl:163);
 *   - the source of photon k is positions[k % npos] (src/kernel.jl:173);
 *   - counts are column-major (nx, ny, nbins+1): counts[i + nx*(j + ny*bin)],
 *     so a Julia Array{UInt32,3} aliases them (src/transport.jl:64-80);
 *   - the record index idx = (jj-1)*nx + ii is 1-based and negative for a
 *     detection on the z = 0 face (src/kernel.jl:232-235).
 *
 * Ownership: the caller owns every host buffer; the library owns device
 * buffers and a CUDA stream inside the opaque handle and reuses them across
 * calls.  No pointer is retained after a call returns.  A handle is not
 * re-entrant: use one handle per host thread.  Errors are returned as
 * negative codes with a message from cl_last_error(); the library never
 * aborts the process.
 */
#ifndef CRYSPLIGHT_CUDA_H
#define CRYSPLIGHT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CL_ABI_VERSION 1

/* Photon fates, src/transport.jl:6-12. */
#define CL_STATUS_DETECTED 1
#define CL_STATUS_ABS_BULK 2
#define CL_STATUS_ABS_WALL 3
#define CL_STATUS_ABS_SIPM 4
#define CL_STATUS_CAP      5
#define CL_STATUS_ABS_SUR  6

/* Return codes.  The reference raises Julia exceptions instead. */
#define CL_OK            0
#define CL_ERR_ARG      -1   /* invalid argument (reference: ArgumentError/BoundsError) */
#define CL_ERR_CUDA     -2   /* CUDA runtime failure                                    */
#define CL_ERR_OOM      -3   /* device allocation failed                                */
#define CL_ERR_TIMEOUT  -4   /* a device-side loop budget ran out                       */
#define CL_ERR_STATE    -5   /* handle misuse (null handle, wrong device)               */

/* Largest max_bounces the transport entry points accept (CL_ERR_ARG above).
 * The reference's default is 100,000 (src/config.jl:68, src/kernel.jl:318);
 * values <= 0 are accepted and, as in the reference (src/transport.jl:140,229),
 * cap every photon at its first wall interaction or scatter. */
#define CL_MAX_BOUNCES_LIMIT 10000000

/* Device time budget of a transport launch on a new handle, in seconds
 * (cl_set_time_budget). */
#define CL_DEFAULT_TIME_BUDGET_S 300.0

/* Box, src/geometry.jl:14-16: crystal [0,L0]x[0,L1]x[0,L2] in mm. */
typedef struct cl_box {
    float L[3];
} cl_box;

/* OpticalParams, src/transport.jl:14-24 (32 bytes). */
typedef struct cl_optical_params {
    float   n_crystal;
    float   n_coupling;
    float   abs_len_mm;     /* +Inf disables bulk absorption     */
    float   rayleigh_mm;    /* +Inf disables Rayleigh scattering */
    float   wrap_R;
    uint8_t wrap_specular;  /* 1 = ESR (specular), 0 = PTFE (Lambertian) */
    uint8_t air_gap;        /* 1 = back-painted, 0 = front-painted      */
    float   sigma_alpha;    /* UNIFIED roughness, radians               */
    float   pde;
} cl_optical_params;

/* SipmGrid, src/transport.jl:26-30 (12 bytes). */
typedef struct cl_sipm_grid {
    float   pitch_mm;
    int32_t nx;
    int32_t ny;
} cl_sipm_grid;

/* Readout, src/transport.jl:41-50 (36 bytes). */
typedef struct cl_readout {
    cl_sipm_grid grid;
    uint8_t disc;           /* 1 = only a disc of radius sqrt(r2) about (cx,cy) is active */
    float   cx;
    float   cy;
    float   r2;
    float   sur_R;
    uint8_t sur_specular;
    uint8_t two_sided;      /* sensors on both z faces */
} cl_readout;

/* TimeBinning, src/transport.jl:59-62: counts have nbins+1 bins, the last one overflow. */
typedef struct cl_time_binning {
    float   bin_ns;
    int32_t nbins;
} cl_time_binning;

/* Scalar fields of Accumulator, src/transport.jl:64-76, same order. */
typedef struct cl_counters {
    int64_t ndet;
    int64_t ndet_front;
    int64_t nabs_bulk;
    int64_t nabs_wall;
    int64_t nabs_sipm;
    int64_t ncap;
    int64_t nabs_sur;
    int64_t nscat;
    int64_t sum_bounces_det;
} cl_counters;

/* Per-photon records of transport_kernel!, src/kernel.jl:159-161,300-303
 * (11 bytes per photon).  Any pointer may be NULL to skip that field. */
typedef struct cl_records {
    uint8_t* status;
    int16_t* idx;
    float*   t;
    int32_t* bounces;
} cl_records;

typedef struct cl_handle cl_handle;

/* Library version string and ABI version (CL_ABI_VERSION). */
const char* cl_version(void);
int cl_abi_version(void);

/* Create a handle bound to CUDA device `device`.  The reference's equivalent
 * is the backend choice ArrayT / KA.get_backend (src/kernel.jl:330). */
int cl_create(cl_handle** out, int device);
void cl_destroy(cl_handle* h);
/* Message of the last failing call on this handle ("" if none).  With a NULL
 * handle, the message of the last failing cl_create or cl_run_photons_noalloc
 * on this thread. */
const char* cl_last_error(const cl_handle* h);

/*
 * Point-source / position-scan transport with host buffers — the replacement
 * for run_photons_ka!(...) (src/kernel.jl:312-367) and, for pid_offset = 0 and
 * pt = NULL, for run_photons! (src/transport.jl:245-273).
 *
 *   px,py,pz   npos source positions (mm); photon k starts at position k % npos
 *   pt         npos emission-time offsets (ns), or NULL for zeros (t0s)
 *   n_photons  number of photons; pid = pid_offset + k + 1
 *   tau_ns     exponential emission time constant, 0 = delta
 *   counts     out: nx*ny*(nbins+1) uint32, column-major (overwritten)
 *   first_ns   out: nx*ny float, earliest detection per SiPM, +Inf if none
 *   counters   out: Accumulator counters
 *   records    optional per-photon records (host arrays of n_photons), or NULL
 *
 * Synchronous.  Results are bit-identical for any launch configuration.
 */
int cl_run_photons(cl_handle* h,
                   const cl_box* box, const cl_optical_params* op,
                   const cl_readout* ro, const cl_time_binning* tb,
                   const float* px, const float* py, const float* pz,
                   const float* pt, int32_t npos,
                   int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                   float tau_ns, int32_t max_bounces,
                   uint32_t* counts, float* first_ns, cl_counters* counters,
                   const cl_records* records);

/*
 * Same as cl_run_photons with every pointer in device memory, enqueued on
 * `stream` (a cudaStream_t; NULL = the handle's own stream, so pass
 * cudaStreamLegacy or cudaStreamPerThread to select a default stream) without
 * a host synchronisation.  `counters` is device memory too.  Call cl_sync() to wait
 * and to collect device-side errors.
 */
int cl_run_photons_device(cl_handle* h,
                          const cl_box* box, const cl_optical_params* op,
                          const cl_readout* ro, const cl_time_binning* tb,
                          const float* d_px, const float* d_py, const float* d_pz,
                          const float* d_pt, int32_t npos,
                          int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                          float tau_ns, int32_t max_bounces,
                          uint32_t* d_counts, float* d_first_ns,
                          cl_counters* d_counters, const cl_records* d_records,
                          void* stream);

/*
 * Segmented transport: many sources, each emitting its own number of photons,
 * grouped into segments (points of a scan, or 511 keV events).  This is the
 * batched form of the event pipeline's flush! (src/events.jl:65-91) and of a
 * per-point scan (one run_photons_ka! call per point with pid_offset =
 * photons before it): photons are numbered source-major, photon k (0-based,
 * over the whole call) has pid = pid_offset + k + 1 and belongs to the source
 * s with src_offsets[s] <= k < src_offsets[s+1], starting at
 * (sx,sy,sz)[s] with emission offset st[s] (NULL = 0).
 *
 *   src_offsets  n_src+1 non-decreasing int64 prefix sums, src_offsets[0] = 0
 *   src_segment  n_src segment ids in [0, n_segments), non-decreasing
 *   maps         out: nx*ny*n_segments uint32, time-integrated detected counts
 *                per segment, maps[i + nx*(j + ny*seg)] (events.jl: maps[ii,jj,ev])
 *   tmin         out: nx*ny*n_segments float, first detection time, +Inf if none
 *   npe          out: n_segments int32, detections per segment
 *   counters     out: totals over the call
 *   records      optional, per photon, indexed by k
 *
 * Host buffers, synchronous.  `tb` is accepted for interface symmetry; the
 * per-segment maps are time-integrated as in the event pipeline.
 */
int cl_run_segments(cl_handle* h,
                    const cl_box* box, const cl_optical_params* op,
                    const cl_readout* ro, const cl_time_binning* tb,
                    const float* sx, const float* sy, const float* sz,
                    const float* st, const int64_t* src_offsets,
                    const int32_t* src_segment, int64_t n_src, int64_t n_segments,
                    uint64_t seed, uint64_t pid_offset,
                    float tau_ns, int32_t max_bounces,
                    uint32_t* maps, float* tmin, int32_t* npe,
                    cl_counters* counters, const cl_records* records);

/* Device-memory, asynchronous form of cl_run_segments (see
 * cl_run_photons_device).  n_photons must equal d_src_offsets[n_src]; the
 * offsets and segment ids are trusted (the host form validates them). */
int cl_run_segments_device(cl_handle* h,
                           const cl_box* box, const cl_optical_params* op,
                           const cl_readout* ro, const cl_time_binning* tb,
                           const float* d_sx, const float* d_sy, const float* d_sz,
                           const float* d_st, const int64_t* d_src_offsets,
                           const int32_t* d_src_segment, int64_t n_src,
                           int64_t n_segments, int64_t n_photons,
                           uint64_t seed, uint64_t pid_offset,
                           float tau_ns, int32_t max_bounces,
                           uint32_t* d_maps, float* d_tmin, int32_t* d_npe,
                           cl_counters* d_counters, const cl_records* d_records,
                           void* stream);

/* cl_run_segments_device plus per-(segment, SiPM) arrival-time moments, the
 * training targets of the light-response surrogate (no counterpart in the
 * reference).  For every detected photon with arrival time t (ns, as in the
 * first-hit times), tc = min(max(t, 0), CL_MOMENT_T_MAX_NS) and
 *   d_tsum [slot] += round(tc * CL_MOMENT_T_SCALE)
 *   d_tsum2[slot] += round(fl(tc * tc) * CL_MOMENT_T2_SCALE)
 * (Float32 products, round to nearest even; slot as in d_maps), so the sums
 * are exact integers independent of the order of the photons.  They cannot
 * overflow below about 1.6e7 detections per slot. */
#define CL_MOMENT_T_SCALE 1048576.0f    /* 2^20 per ns */
#define CL_MOMENT_T2_SCALE 65536.0f     /* 2^16 per ns^2 */
#define CL_MOMENT_T_MAX_NS 4096.0f
int cl_run_segments_moments_device(cl_handle* h,
                                   const cl_box* box, const cl_optical_params* op,
                                   const cl_readout* ro, const cl_time_binning* tb,
                                   const float* d_sx, const float* d_sy, const float* d_sz,
                                   const float* d_st, const int64_t* d_src_offsets,
                                   const int32_t* d_src_segment, int64_t n_src,
                                   int64_t n_segments, int64_t n_photons,
                                   uint64_t seed, uint64_t pid_offset,
                                   float tau_ns, int32_t max_bounces,
                                   uint32_t* d_maps, float* d_tmin, int32_t* d_npe,
                                   cl_counters* d_counters, uint64_t* d_tsum, uint64_t* d_tsum2,
                                   void* stream);

/*
 * Events from the learned light-response surrogate with Monte Carlo fallback
 * (no counterpart in the reference: it replaces, for the deposits the
 * surrogate is trusted with, the transport that flush! (src/events.jl:65-91)
 * launches through run_photons_ka!).  One call, all on `stream`:
 *   1. the deposits that fell back to the Monte Carlo are transported exactly
 *      as by cl_run_segments_device (same source, offset and segment arrays,
 *      n_src may be 0);
 *   2. every site i with d_site_flag[i] == 0 (d_site_flag may be NULL) splits
 *      its d_site_photons[i] photons over the nx*ny SiPMs multinomially with
 *      the per-photon detection probabilities d_site_p[i][cell] (conditional
 *      binomial draws) and draws each hit SiPM's first-hit time as the minimum
 *      of its photons' arrival times d_site_t0[i] + Exp(tau_ns) +
 *      N(d_site_tmean, d_site_tsig^2); counts and times join segment
 *      d_site_segment[i]'s map;
 *   3. the maps' first times are decoded and npe summed, as in segment mode.
 * Sampler uniforms: Philox4x32-10 keyed by sample_seed, a stream per site.
 * d_counters count the Monte Carlo photons only; d_sampled (uint64[2], may be
 * NULL) gets the photons of sampled sites and their sampled detections.
 * Asynchronous; cl_sync reports CL_ERR_TIMEOUT if a sampler loop budget ran
 * out and CL_ERR_ARG if a sampled site's segment id lay outside
 * [0, n_segments) (that site is skipped).
 */
int cl_run_events_surrogate_device(cl_handle* h,
                                   const cl_box* box, const cl_optical_params* op,
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
                                   cl_counters* d_counters, uint64_t* d_sampled, void* stream);

/*
 * Ensemble reduction of the surrogate (no counterpart in the reference).
 * d_raw [members][n_sites][3*64]: each member's standardised outputs
 * (cl_mlp_forward); y = raw * d_y_std + d_y_mean gives per SiPM (64 = nx*ny,
 * required) log detection probability, mean transit time (ns) and log of its
 * standard deviation.  Writes per site and SiPM d_p = pde * mean_k exp(log p),
 * d_tmean = mean_k, d_tsig = exp(mean_k log sigma); d_spread = sum over SiPMs
 * of the members' standard deviation of p / sum of their mean p; d_flag bit 0:
 * spread > spread_max, bit 1: the site (d_xyz [n][3] mm) lies closer than
 * wall_min_mm to a wrapped face (the four side faces and, unless two-sided,
 * the front face z = 0), bit 2: pde * sum of p >= 0.999.  Asynchronous on
 * `stream`; allocates nothing.
 */
int cl_surrogate_combine(const float* d_raw, int32_t members, int64_t n_sites,
                         const float* d_y_mean, const float* d_y_std, const float* d_xyz,
                         const cl_box* box, const cl_readout* ro, float pde,
                         float spread_max, float wall_min_mm,
                         float* d_p, float* d_tmean, float* d_tsig, float* d_spread,
                         uint8_t* d_flag, void* stream);

/*
 * As cl_surrogate_combine, with d_direct [n_sites][64] (device, may be NULL):
 * the sites' first-pass probabilities (cl_surrogate_direct) for an ensemble
 * trained on the light response minus that term.  They are added to the
 * members' mean before the PDE (d_p = pde * (d_direct + mean_k p_k)) and to
 * the total the spread is relative to (d_spread = sum of the members'
 * standard deviations / sum of (d_direct + mean_k p_k)); the members' spread
 * itself does not include them.  No counterpart in the reference.
 */
int cl_surrogate_combine_direct(const float* d_raw, int32_t members, int64_t n_sites,
                                const float* d_y_mean, const float* d_y_std, const float* d_xyz,
                                const float* d_direct, const cl_box* box, const cl_readout* ro, float pde,
                                float spread_max, float wall_min_mm,
                                float* d_p, float* d_tmean, float* d_tsig, float* d_spread,
                                uint8_t* d_flag, void* stream);

/*
 * First-pass light of n_sites emission points (no counterpart in the
 * reference): d_out[i][c] = probability that a photon emitted isotropically
 * at d_xyz[i] (mm) reaches the readout face z = Lz without a bulk interaction
 * (absorption or Rayleigh scattering: survival exp(-d (1/abs_len +
 * 1/rayleigh)) over the path d), is transmitted by the face (the Fresnel
 * coefficients of the transport, n_crystal -> n_coupling, total internal
 * reflection beyond the critical angle) and lands in SiPM c's pixel, at
 * PDE 1; landing points off the face count for nothing (those photons meet a
 * side wall first).  Computed by quadrature over the polar angle (64
 * Gauss-Legendre nodes up to the critical angle) with the azimuthal arcs of
 * each pixel exact.  Requires a 64-cell grid read out on the face z = Lz
 * only (no disc, not two-sided).  Device arrays, asynchronous on `stream`;
 * allocates nothing.
 */
int cl_surrogate_direct(const float* d_xyz, int64_t n_sites, const cl_box* box, const cl_optical_params* op,
                        const cl_readout* ro, float* d_out, void* stream);

/*
 * Network inputs of the surrogate for n_sites emission points (no counterpart
 * in the reference): d_out[i] = (2x/Lx - 1, 2y/Ly - 1, 2w - 1) for
 * d_xyz[i] = (x, y, z) in mm, with the depth warp
 * w = (1 - z_warp) t + z_warp (1 - sqrt(1 - t)), t = z/Lz clamped to [0, 1]
 * (z_warp in [0, 1]; the readout face is z = Lz).  Device arrays [n][3],
 * asynchronous on `stream`; allocates nothing.
 */
int cl_surrogate_inputs(const float* d_xyz, int64_t n_sites, const cl_box* box, float z_warp,
                        float* d_out, void* stream);

/*
 * Diagnostics for tests: n draws (stream i = draw i, key = seed) of the
 * surrogate sampler's variates into device memory: fn 0 = binomial
 * (n = par[0], p = par[1]) -> int64; fn 1 = minimum of k = par[0] arrival
 * times Exp(tau = par[3]) + N(mu = par[1], sigma = par[2]^2) -> double.
 * *d_err (device, may be NULL) gets bit 2 if a loop budget ran out.
 */
int cl_debug_sampler(int fn, const double* par, int64_t n, uint64_t seed, void* d_out,
                     unsigned int* d_err, void* stream);

/* Wait for the work enqueued by the *_device calls on `stream` (NULL = the
 * handle's stream) and report device-side errors (CL_ERR_TIMEOUT). */
int cl_sync(cl_handle* h, void* stream);

/*
 * Number of transport-loop iterations ("photon-steps": wall interactions,
 * Rayleigh scatters and terminal steps) executed by the last completed call on
 * this handle.  Diagnostic for throughput per step; 0 if not available.
 */
int64_t cl_last_steps(const cl_handle* h);

/*
 * Launch shape used by the transport kernels: CTAs per SM and threads per CTA
 * (0 = automatic), and the number of photons a warp claims from the device
 * work queue at a time.  Results do not depend on these values.
 */
int cl_set_launch(cl_handle* h, int ctas_per_sm, int threads_per_cta,
                  int warp_chunk);

/*
 * Device-side time budget of every transport launch on this handle: the
 * kernel's warps stop once the launch has run `seconds` of wall-clock time on
 * the GPU, and the call (or cl_sync for the *_device calls) returns
 * CL_ERR_TIMEOUT; the outputs of such a call are incomplete.  It bounds the
 * time a launch can hold a shared GPU whatever n_photons x max_bounces is
 * (photons trapped by total internal reflection in an ideal reflector bounce
 * until max_bounces).  0 = no budget; default CL_DEFAULT_TIME_BUDGET_S.  The
 * reference has no counterpart (its loop is bounded by max_bounces alone,
 * src/transport.jl:228-232).  CL_ERR_ARG for a negative or non-finite value.
 */
int cl_set_time_budget(cl_handle* h, double seconds);

/*
 * Diagnostics for tests: evaluate the device's Float32 elementary functions
 * on n inputs.  fn: 0 = log, 1 = sin, 2 = cos, 3 = Philox4x32-10 on
 * (in_u32[4k..4k+3] counter, key = (seed lo, hi)) -> out_u32[4k..4k+3],
 * 4 = randu stream: out[k*m + i] = i-th uniform of pid = k + 1 (m = n_per),
 * 5 = cuRAND's Philox4x32-10 on the same inputs as 3 (cross-check),
 * 6 = the first n entries of the handle's table of logs of the uniforms,
 * out_f32[k] = log((k+1) * 2^-24) as the transport uses it (in unused).
 * Host buffers, synchronous.
 */
int cl_debug_eval(cl_handle* h, int fn, const void* in, void* out, int64_t n,
                  uint64_t seed, int32_t n_per);

/*
 * Diagnostic for tests: C = A * B^T on the tcgen05 tensor cores, A [M][K] and
 * B [N][K] BF16 row-major device arrays, C [M][N] FP32 device (or, with
 * splits > 1, K-split partials C[split][M][N]).  M % 128 == 0, N % 32 == 0,
 * N <= 256, K % 64 == 0.  *d_err (device) gets bit 0 set if a completion wait
 * ran out.  Enqueued on `stream`; no synchronisation.
 */
int cl_umma_gemm_bf16(const void* A, const void* B, float* C, int M, int N, int K,
                      int grid_x, int splits, unsigned int* d_err, void* stream);

/* ---------------------------------------------------------------------------
 * Light-response surrogate network (no counterpart in the reference, which
 * always runs the Monte Carlo): a 3 -> 256 -> 256 -> 256 -> 192 SiLU MLP
 * trained and evaluated on the tcgen05 tensor cores (BF16 weights and
 * activations, FP32 accumulation, Adam on FP32 master weights).  Parameters
 * are one FP32 block of cl_mlp_param_count() floats:
 * W1[256][3] b1[256] W2[256][256] b2[256] W3[256][256] b3[256] W4[192][256] b4[192]
 * (W[out][in]).  A cl_mlp owns one stream and is not re-entrant.
 * ------------------------------------------------------------------------- */
typedef struct cl_mlp cl_mlp;

int cl_mlp_param_count(void);
/* max_batch % 128 == 0; parameters start at zero (set them before use). */
int cl_mlp_create(cl_mlp** out, int device, int max_batch);
void cl_mlp_destroy(cl_mlp* m);
const char* cl_mlp_last_error(const cl_mlp* m);
/* Cap the CTAs of the batch-tiled GEMMs (0 = one per SM), for tests. */
int cl_mlp_set_max_ctas(cl_mlp* m, int n);
/* Host buffers of cl_mlp_param_count() floats; setting resets Adam's state. */
int cl_mlp_set_params(cl_mlp* m, const float* host);
int cl_mlp_get_params(cl_mlp* m, float* host);
/* Training set x [n][3], targets t [n][192]: FP32 device arrays owned by the
 * caller, alive across the cl_mlp_train calls. */
int cl_mlp_set_data(cl_mlp* m, const float* d_x, const float* d_t, int64_t n);
/* `steps` Adam steps (lr, betas 0.9/0.999) on minibatches of `batch` rows
 * (batch % 128 == 0, <= max_batch) drawn with replacement by Philox from
 * (seed, step0 + s); loss = mean squared error over all 192 outputs.
 * *loss_out = mean loss over the steps. */
int cl_mlp_train(cl_mlp* m, int steps, int batch, float lr, uint32_t seed, uint32_t step0,
                 float* loss_out);
/* Inference: out [n][192] FP32 device for x [n][3] FP32 device. */
int cl_mlp_forward(cl_mlp* m, const float* d_x, float* d_out, int64_t n);
/* Loss and gradient (host, cl_mlp_param_count() floats) for one batch of
 * B rows (B % 128 == 0, <= max_batch), without an update.  For tests. */
int cl_mlp_gradient(cl_mlp* m, const float* d_x, const float* d_t, int B, float* host_grad,
                    float* loss_out);

/* ---------------------------------------------------------------------------
 * Host-side 511 keV gamma stage of the event pipeline (no GPU involved).
 * The reference runs it in Julia (its vendored gamma core, the src/gamma files,
 * through src/gamma_interface.jl); these restate it in C.  Each event draws
 * from its own Philox4x32-10 stream keyed by (seed, event number), so the
 * gamma stage is statistically, not bitwise, equivalent to the reference
 * (whose Julia Xoshiro stream cannot be reproduced here).
 * ------------------------------------------------------------------------- */
typedef struct cl_gamma_material cl_gamma_material;

/* make_material(name, density, xcom_csv) (src/gamma/gmaterials.jl:22-31):
 * XCOM columns in cm^2/g at n energies (MeV, duplicate K-edge energies
 * allowed), density in g/cm^3.  n = 0 gives the vacuum material. */
int cl_gamma_material_create(cl_gamma_material** out, const double* E_MeV,
                             const double* incoherent, const double* photoelectric,
                             const double* pair_nuclear, const double* pair_electron,
                             int32_t n, double density);
void cl_gamma_material_destroy(cl_gamma_material* m);
const char* cl_gamma_last_error(void);

/* sigma_macro (src/gamma/gmaterials.jl:45-57): sigma3 = (Compton,
 * photoelectric, pair) macroscopic cross sections in 1/cm at E_MeV. */
int cl_gamma_sigma(const cl_gamma_material* m, double E_MeV, double* sigma3);

/* gamma_deposits (src/gamma_interface.jl:30-49) for one gamma entering the
 * crystal at entry_mm along dir, drawing from stream `stream` of `seed`:
 * dep6[6*i..] = (x, y, z [mm], E [keV], t [ns], process 0 photo / 1 Compton /
 * 2 below the 10 keV cut). */
int cl_gamma_deposits(const cl_gamma_material* m, const cl_box* box, const float* entry_mm,
                      const double* dir, double e0_mev, uint64_t seed, uint64_t stream,
                      float* dep6, int32_t max_dep, int32_t* n_dep);

/* rand_poisson (src/events.jl:11-22) drawing from stream `stream` of `seed`. */
int64_t cl_rand_poisson(uint64_t seed, uint64_t stream, double lam);

/*
 * The gamma half of run_events! (src/events.jl:93-118) for events
 * ev0+1 .. ev0+n_events (1-based event numbers key the streams): per event
 * the entry point uniform on z = 0, the deposits, the truth record (edep,
 * xyz1[3], e1, xyz2[3], e2, er [keV / mm], int_type, n_int) and, per deposit
 * in event order, its position, time, event index (0-based within the call)
 * and Poisson photon count for yield_per_mev.  Deposits beyond max_deposits
 * give CL_ERR_ARG with *n_deposits set to the number needed.  nthreads <= 0
 * uses every hardware thread; results do not depend on it.
 */
int cl_gamma_events(const cl_gamma_material* m, const cl_box* box, int64_t ev0,
                    int64_t n_events, uint64_t seed, double e0_mev, double yield_per_mev,
                    int nthreads, float* edep, float* xyz1, float* e1, float* xyz2,
                    float* e2, float* er, int8_t* int_type, int16_t* n_int,
                    int64_t max_deposits, float* dep_xyz, float* dep_t,
                    int32_t* dep_event, int64_t* dep_photons, int64_t* n_deposits);

/*
 * Allocation-free point-source transport.  No counterpart in the reference:
 * it exists for callers that cannot let a library call cudaMalloc — programs
 * whose device memory is owned by a pool or caching allocator (CUDA.jl's,
 * PyTorch's) or by a fixed budget, where a foreign cudaMalloc can fail or
 * break the accounting, and latency-sensitive loops where cudaMalloc/cudaFree
 * would synchronise the device.
 *
 * Same arguments and results as cl_run_photons with host buffers, minus the
 * handle and the per-photon records.  All device-side memory it uses —
 * staged source positions, the count histogram, first-time keys, counters and
 * the work-queue words — lives in one file-scope device array of
 * CL_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * process exit.  The staged data is 512 bytes of queue words and counters
 * plus four float arrays of npos, nx*ny*(nbins+1) count words and nx*ny key
 * words, each array rounded up to a multiple of 256 bytes; calls where that
 * exceeds CL_NOALLOC_SCRATCH_BYTES (1 MiB: e.g. an 8x8 grid with up to about
 * 4000 time bins) return CL_ERR_ARG with a message from cl_last_error(NULL).
 * The function calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * Runs on the current CUDA device and on `stream` (NULL = the legacy default
 * stream), and synchronises that stream before returning.  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) and
 * caches it; make that first call before any stream capture.  Every call
 * shares the one array and overwrites it, so calls that overlap on the GPU
 * (other host threads, other streams) race: serialise them.
 */
#define CL_NOALLOC_SCRATCH_BYTES (1u << 20)

int cl_run_photons_noalloc(const cl_box* box, const cl_optical_params* op,
                           const cl_readout* ro, const cl_time_binning* tb,
                           const float* px, const float* py, const float* pz,
                           const float* pt, int32_t npos,
                           int64_t n_photons, uint64_t seed, uint64_t pid_offset,
                           float tau_ns, int32_t max_bounces,
                           uint32_t* counts, float* first_ns, cl_counters* counters,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CRYSPLIGHT_CUDA_H */
