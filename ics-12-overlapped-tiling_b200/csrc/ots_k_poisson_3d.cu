// Kernel instantiations for poisson-3d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_poisson_3d() {
  static const StencilKernels k = make_kernels_with_stream<OpPoisson3D>();
  return k;
}
}  // namespace ots
