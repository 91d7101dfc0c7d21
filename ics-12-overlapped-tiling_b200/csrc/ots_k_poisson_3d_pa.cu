// Packed-FP32 stream kernel instantiations for poisson-3d, E = 4 shapes (a
// translation unit of their own so the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
void fill_stream3p_poisson_3d_a(StencilKernels& k) {
  fill_stream3p_shape<OpPoisson3D, 0>(k, std::make_integer_sequence<int, kMaxT3p>{});
  fill_stream3p_shape<OpPoisson3D, 1>(k, std::make_integer_sequence<int, kMaxT3p>{});
  fill_stream3p_shape<OpPoisson3D, 2>(k, std::make_integer_sequence<int, kMaxT3p>{});
}
}  // namespace ots
