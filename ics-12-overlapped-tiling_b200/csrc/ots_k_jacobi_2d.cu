// Kernel instantiations for jacobi-2d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_jacobi_2d() {
  static const StencilKernels k = make_kernels<OpJacobi2D>();
  return k;
}
}  // namespace ots
