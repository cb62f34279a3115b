// Kernel table shared by the host code and the two instantiation units.
#pragma once

namespace cgpu {

struct DevProg;
struct KParams;
using KernelFn = void (*)(const DevProg, const KParams);

// G = lanes per shot (1, 2, 4, 8, 16, 32), 0 for one CTA per shot, -1 for
// one CTA per shot whose last warp moves the fused blocks' tiles;
// nw = frame words (1, or 2..4 served by the 4-word kernel); dense (G <= 0):
// the instance with the tensor-core dense blocks.
KernelFn kernel_f32(int G, int nw, bool dense = false);
KernelFn kernel_f64(int G, int nw);

}  // namespace cgpu
