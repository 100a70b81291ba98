// cl_surrogate.cuh — host-side interface between the transport library and
// the surrogate event sampler (cl_surrogate.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cl {

// One launch of the surrogate site sampler: every site with flag == 0 adds
// its sampled SiPM counts and first-hit-time keys to its segment's slots of
// `maps` / `keys` (the layout of the segment-mode transport before its
// finalize pass).
struct SurSampleArgs {
    const float* p;          // [n][cells] detection probability per photon
    const float* tmean;      // [n][cells] mean transit time (ns)
    const float* tsig;       // [n][cells] transit-time standard deviation (ns)
    const uint8_t* flag;     // [n] nonzero: the site went to the Monte Carlo (may be NULL)
    const float* t0;         // [n] deposit time (ns)
    const int64_t* photons;  // [n] photons emitted by the site
    const int32_t* seg;      // [n] segment (event) index
    int64_t n;
    int64_t n_seg;           // segments in maps / keys (sites outside are skipped, bit 3 of err)
    int32_t cells;
    uint32_t k0, k1;         // Philox key (seed)
    float tau;               // scintillation decay time (ns), 0 = prompt
    uint32_t* maps;          // [n_seg][cells] counts
    uint32_t* keys;          // [n_seg][cells] order-preserving time keys
    unsigned long long* stats;  // [2] += photons of sampled sites, sampled detections (may be NULL)
    unsigned int* err;       // bit 2: a sampler loop budget ran out; bit 3: a segment id out of range
};

// Enqueue the sampler on `st`; returns a cudaError_t of the launch.
cudaError_t launch_surrogate_sample(const SurSampleArgs& a, int num_sms, cudaStream_t st);

}  // namespace cl
