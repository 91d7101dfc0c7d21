// Kernel instantiations for fdtd-2d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_fdtd_2d() {
  static const StencilKernels k = make_kernels<OpFdtd2D>();
  return k;
}
}  // namespace ots
