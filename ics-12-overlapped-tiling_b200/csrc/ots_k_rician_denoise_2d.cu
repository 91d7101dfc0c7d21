// Kernel instantiations for rician-denoise-2d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_rician_denoise_2d() {
  static const StencilKernels k = make_kernels<OpRician2D>();
  return k;
}
}  // namespace ots
