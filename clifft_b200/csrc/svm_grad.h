// svm_grad.h -- launch parameters of the adjoint expectation-value gradient
// kernel (svm_grad.cu), shared with the host side (clifft_gpu.cu).
#pragma once

#include <cstdint>

namespace cgpu {

struct DevProg;

struct GradParams {
    uint64_t batch;            // parameter vectors
    uint32_t n_exp;            // EXP_VAL instructions (one task each per vector)
    uint32_t n_out;            // rows of the output (num_exp_vals)
    uint32_t n_params;         // ARRAY_ROT / EXPAND_ROT instructions
    const int32_t* rot_index;  // per instruction: its parameter index, or -1
    const uint32_t* exp_pc;    // per EXP_VAL: instruction index
    const uint32_t* exp_out;   // per EXP_VAL: output row
    const double* phases;      // batch x n_params rotation phases (radians), or null = the payloads
    void* slab;                // per resident CTA: two 2^peak statevectors (v, lambda)
    uint64_t stride;           // 2^peak
    unsigned long long* work;  // task counter
    double* out_exp;           // batch x n_out
    double* out_grad;          // batch x n_out x n_params
};

using ExpvalGradFn = void (*)(const DevProg, const GradParams);
ExpvalGradFn expval_grad_kernel_fn(bool fp32);
constexpr int kExpvalGradThreads = 256;

}  // namespace cgpu
