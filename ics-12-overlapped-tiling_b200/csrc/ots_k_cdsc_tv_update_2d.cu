// Kernel instantiations for cdsc-tv-update-2d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_cdsc_tv_update_2d() {
  static const StencilKernels k = make_kernels<OpTvUpdate2D>();
  return k;
}
}  // namespace ots
