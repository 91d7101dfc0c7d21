// Kernel instantiations for jacobi-3d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_jacobi_3d() {
  static const StencilKernels k = make_kernels_with_stream<OpJacobi3D>();
  return k;
}
}  // namespace ots
