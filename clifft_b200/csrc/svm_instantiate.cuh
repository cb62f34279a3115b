// Kernel-table construction for one statevector precision.
#pragma once
#include "svm_dispatch.h"
#include "svm_kernel.cuh"

namespace cgpu {
template <typename R, int NW>
KernelFn pick_by_group(int G) {
    switch (G) {
        case 1: return svm_sample_kernel<R, 1, NW>;
        case 2: return svm_sample_kernel<R, 2, NW>;
        case 4: return svm_sample_kernel<R, 4, NW>;
        case 8: return svm_sample_kernel<R, 8, NW>;
        case 16: return svm_sample_kernel<R, 16, NW>;
        case 32: return svm_sample_kernel<R, 32, NW>;
        case -1: return svm_sample_kernel<R, -1, NW>;
        default: return svm_sample_kernel<R, 0, NW>;
    }
}
template <typename R>
KernelFn pick_kernel_impl(int G, int nw) {
    return nw <= 1 ? pick_by_group<R, 1>(G) : pick_by_group<R, 4>(G);
}
}  // namespace cgpu
