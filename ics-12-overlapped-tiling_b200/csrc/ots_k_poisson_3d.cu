// Kernel instantiations for poisson-3d (one translation unit per stencil so
// the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_poisson_3d() {
  static const StencilKernels k = [] {
    StencilKernels t = make_kernels_with_stream<OpPoisson3D>();
    fill_stream3p_poisson_3d_a(t);  // the packed-FP32 stream kernel (star form)
    fill_stream3p_poisson_3d_b(t);
    return t;
  }();
  return k;
}
}  // namespace ots
