// svm_sample_k.cu -- fault-set draws for k-fault importance sampling
// (src/clifft/svm/svm.cc:356-711, clifft::sample_k / sample_k_survivors).
//
// Each shot conditions on exactly k fault events among the quantum noise
// sites and readout entries. One thread per shot draws the set from its own
// Philox stream (stream 1 of the shot's counter space, apart from the
// executor's stream 0):
//  * general case: the exact conditional Poisson-binomial distribution, site
//    by site in index order, including site i with probability
//    w_i * DP[i+1][j-1] / DP[i][j] (j faults still needed; DP[i][j] the sum of
//    products of odds ratios w over the size-j subsets of sites i..N-1);
//  * equal probabilities: a uniform k-subset (Floyd's algorithm), the same
//    distribution the reference draws with a persistent Fisher-Yates pool.
// A fired quantum site's channel is drawn as the executor's NOISE opcode
// draws it (a uniform times the site's probability sum against the running
// channel sum); the executor then replays the set as forced faults.

#include <cuda_runtime.h>

#include "svm_kernel.cuh"
#include "svm_sample_k.h"

namespace cgpu {

namespace {

__global__ void __launch_bounds__(256) sample_k_prepare_kernel(const DevProg P, const SampleKParams S) {
    const uint32_t k = S.k;
    for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < S.shots;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t gshot = S.first_shot + s;
        uint32_t draw = 0;
        const uint64_t base = s * k;
        uint32_t nq = 0, nr = 0;
        auto take = [&](uint32_t idx) {
            if (idx < S.n_q) {
                const uint32_t c0 = __ldg(P.site_off + idx), c1 = __ldg(P.site_off + idx + 1);
                const double r = philox_uniform(S.seed, gshot, draw++, 1u) * __ldg(P.site_psum + idx);
                double cum = 0.0;
                uint32_t c = c0;
                for (; c < c1; ++c) {
                    cum += __ldg(P.chan_prob + c);
                    if (r < cum) break;
                }
                S.fault_sites[base + nq] = idx;
                S.fault_chan[base + nq] = c - c0;  // == channel count: no channel fires
                ++nq;
            } else {
                S.ro_entries[base + nr] = idx - S.n_q;
                ++nr;
            }
        };
        if (S.uniform) {
            uint32_t chosen[kSampleKUniformMax];
            uint32_t m = 0;
            for (uint32_t j = S.n_total - k; j < S.n_total; ++j) {
                const double u = philox_uniform(S.seed, gshot, draw++, 1u);
                uint32_t t = (uint32_t)(u * (double)(j + 1));
                if (t > j) t = j;
                bool dup = false;
                for (uint32_t q = 0; q < m; ++q) dup |= chosen[q] == t;
                const uint32_t pick = dup ? j : t;
                // insertion into the sorted prefix
                uint32_t q = m++;
                while (q > 0 && chosen[q - 1] > pick) {
                    chosen[q] = chosen[q - 1];
                    --q;
                }
                chosen[q] = pick;
            }
            for (uint32_t q = 0; q < m; ++q) take(chosen[q]);
        } else {
            const uint32_t stride = k + 1;
            uint32_t needed = k;
            for (uint32_t i = 0; i < S.n_total && needed > 0; ++i) {
                double inc;
                if (needed == S.n_total - i) {
                    inc = 1.0;
                } else {
                    const double denom = __ldg(S.dp + (size_t)i * stride + needed);
                    inc = denom > 0.0 ? __ldg(S.w + i) * __ldg(S.dp + (size_t)(i + 1) * stride + (needed - 1)) / denom
                                      : 0.0;
                }
                if (philox_uniform(S.seed, gshot, draw++, 1u) < inc) {
                    take(i);
                    --needed;
                }
            }
        }
        S.fault_off[s] = (uint32_t)base;
        S.fault_end[s] = (uint32_t)base + nq;
        S.ro_off[s] = (uint32_t)base;
        S.ro_end[s] = (uint32_t)base + nr;
    }
}

}  // namespace

void launch_sample_k_prepare(const DevProg& P, const SampleKParams& S, void* stream) {
    const uint64_t blocks = (S.shots + 255) / 256;
    sample_k_prepare_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0,
                              static_cast<cudaStream_t>(stream)>>>(P, S);
}

}  // namespace cgpu
