// Kernel instantiations for jacobi-1d-7pt (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_jacobi_1d_7pt() {
  static const StencilKernels k = make_kernels<OpJacobi1D7>();
  return k;
}
}  // namespace ots
