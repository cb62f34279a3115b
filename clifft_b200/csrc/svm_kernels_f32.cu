// Instantiates the FP32-statevector interpreter kernels (one per shot-group
// width G and frame width NW); see svm_kernel.cuh.
#include "svm_instantiate.cuh"

namespace cgpu {
// FP32 one-CTA-per-shot kernels with the tensor-core dense blocks
static KernelFn pick_dense_f32(int G, int nw) {
    if (G < 0) return nw <= 1 ? svm_sample_kernel<float, -1, 1, true> : svm_sample_kernel<float, -1, 4, true>;
    return nw <= 1 ? svm_sample_kernel<float, 0, 1, true> : svm_sample_kernel<float, 0, 4, true>;
}
KernelFn kernel_f32(int G, int nw, bool dense) {
    return dense && G <= 0 ? pick_dense_f32(G, nw) : pick_kernel_impl<float>(G, nw);
}
}  // namespace cgpu
