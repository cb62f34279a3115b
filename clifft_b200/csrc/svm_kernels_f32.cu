// Instantiates the FP32-statevector interpreter kernels (one per shot-group
// width G and frame width NW); see svm_kernel.cuh.
#include "svm_instantiate.cuh"

namespace cgpu {
KernelFn kernel_f32(int G, int nw) { return pick_kernel_impl<float>(G, nw); }
}  // namespace cgpu
