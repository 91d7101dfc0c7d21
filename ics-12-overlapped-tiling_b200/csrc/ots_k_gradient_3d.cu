// Kernel instantiations for gradient-3d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_gradient_3d() {
  static const StencilKernels k = make_kernels_with_stream<OpGradient3D>();
  return k;
}
}  // namespace ots
