// svm_sample_k.h -- per-shot fault-set draws of k-fault importance sampling
// (clifft_gpu_sample_k), shared by svm_sample_k.cu and clifft_gpu.cu.
#pragma once

#include <cstdint>

namespace cgpu {

struct DevProg;

struct SampleKParams {
    uint64_t shots;
    uint64_t first_shot;
    uint64_t seed;
    uint32_t k;          // faults per shot
    uint32_t n_total;    // quantum noise sites + readout entries
    uint32_t n_q;        // quantum noise sites (indices below n_q)
    uint32_t uniform;    // all probabilities equal: uniform k-subsets
    const double* w;     // DP mode: odds ratios (mean 1)
    const double* dp;    // DP mode: (n_total + 1) x (k + 1), suffix subset-weight sums
    // outputs, stride k per shot
    uint32_t* fault_off;
    uint32_t* fault_end;
    uint32_t* fault_sites;
    uint32_t* fault_chan;
    uint32_t* ro_off;
    uint32_t* ro_end;
    uint32_t* ro_entries;
};

constexpr uint32_t kSampleKUniformMax = 64;  // uniform mode keeps the subset in registers up to this k
void launch_sample_k_prepare(const DevProg& P, const SampleKParams& S, void* stream);

}  // namespace cgpu
