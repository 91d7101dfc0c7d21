// Packed-FP32 stream kernel instantiations for poisson-3d, E = 2 shapes (a
// translation unit of their own so the sm_100a build parallelises).
#include "ots_launch.cuh"

namespace ots {
void fill_stream3p_poisson_3d_b(StencilKernels& k) {
  fill_stream3p_shape<OpPoisson3D, 3>(k, std::make_integer_sequence<int, kMaxT3p>{});
  fill_stream3p_shape<OpPoisson3D, 4>(k, std::make_integer_sequence<int, kMaxT3p>{});
  fill_stream3p_shape<OpPoisson3D, 5>(k, std::make_integer_sequence<int, kMaxT3p>{});
}
}  // namespace ots
