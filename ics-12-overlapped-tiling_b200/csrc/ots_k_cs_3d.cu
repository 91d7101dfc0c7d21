// Kernel instantiations for cs-3d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_cs_3d() {
  static const StencilKernels k = make_kernels<OpCs3D>();
  return k;
}
}  // namespace ots
