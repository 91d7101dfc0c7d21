// ots_launch.cuh -- host launchers and per-stencil kernel tables.
//
// Every kernel is a template instantiation compiled ahead of time for
// sm_100a (E, T and the stencil are template arguments); a plan picks its
// instantiation from these tables, which is what replaces the reference's
// per-run OpenCL source generation and JIT build
// (opencl/jacobi-2d/jacobi-2d.cpp:162-173, 741-780).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "ots_stream.cuh"
#include "ots_stream2d.cuh"
#include "ots_stream3p.cuh"
#include "ots_stream1d.cuh"
#include "ots_tile.cuh"

namespace ots {

constexpr int kMaxE = 16;       // tile kernel, 1D/2D
constexpr int kMaxE3 = 8;       // tile kernel, 3D
constexpr int kMaxT = 8;        // stream kernel levels
constexpr int kStreamEs[3] = {1, 2, 4};
constexpr int kTexMaxE = 8;     // texture-path tile kernel (2D, one state field)

using TileLaunch = cudaError_t (*)(const StepParams&, dim3, dim3, size_t, cudaStream_t);
using StreamLaunch = cudaError_t (*)(const CUtensorMap&, const StreamParams&, dim3, dim3, size_t,
                                     cudaStream_t);
using AttrFn = cudaError_t (*)(cudaFuncAttributes*);
using Stream2dLaunch = cudaError_t (*)(const Stream2dParams&, dim3, cudaStream_t);
using Stream2dgLaunch = cudaError_t (*)(const Stream2dgParams&, dim3, cudaStream_t);
constexpr int kMaxTg = 6;  // generic 2D stream kernel levels
using Stream1dLaunch = cudaError_t (*)(const Stream1dParams&, dim3, cudaStream_t);
constexpr int kStream1dVs[3] = {4, 8, 16};  // cells per lane of the 1D register kernel
using Occ2dFn = cudaError_t (*)(int*);
// the generic 2D stream kernels: `fast` selects the fast-division
// instantiation where an op has one (Rician)
using Occ2dgFn = cudaError_t (*)(int*, bool fast);
using Attr2dgFn = cudaError_t (*)(cudaFuncAttributes*, bool fast);
// stream kernel queries take the cluster flag (the clustered instantiation)
using StreamAttrFn = cudaError_t (*)(cudaFuncAttributes*, bool);
using StreamOccFn = cudaError_t (*)(int*, int, size_t, bool);
using Occ3pFn = cudaError_t (*)(int*, int, size_t);
constexpr int kMaxT3p = 4;  // packed 3D stream kernel levels

struct StencilKernels {
  TileLaunch tile[3][kMaxE + 1] = {};  // [E axis][E]
  AttrFn tile_attr[3][kMaxE + 1] = {};
  TileLaunch plain = nullptr;
  AttrFn plain_attr = nullptr;
  TileLaunch tex[kTexMaxE + 1] = {};  // [E]
  AttrFn tex_attr[kTexMaxE + 1] = {};
  StreamLaunch stream[kMaxT + 1][3] = {};  // [T][index of E in kStreamEs]
  StreamAttrFn stream_attr[kMaxT + 1][3] = {};
  StreamOccFn stream_occ[kMaxT + 1][3] = {};
  bool has_stream = false;
  // packed-FP32 3D stream kernel (ots_stream3p.cuh): [T <= kMaxT3p][shape
  // index in kShape3p]
  StreamLaunch stream3p[kMaxT3p + 1][kShapes3p] = {};
  AttrFn stream3p_attr[kMaxT3p + 1][kShapes3p] = {};
  Occ3pFn stream3p_occ[kMaxT3p + 1][kShapes3p] = {};
  Stream2dLaunch stream2d[kMaxT + 1] = {};  // [T], 2D star stencils
  // packed-FP32 form of the 2D star kernel (Jacobi-2D, Poisson-2D; n0 % 4 == 0)
  Stream2dLaunch stream2dp[kMaxT + 1] = {};
  AttrFn stream2dp_attr[kMaxT + 1] = {};
  Occ2dFn stream2dp_occ[kMaxT + 1] = {};
  AttrFn stream2d_attr[kMaxT + 1] = {};
  Occ2dFn stream2d_occ[kMaxT + 1] = {};
  Stream2dgLaunch stream2dg[kMaxTg + 1] = {};  // [T], any 2D stencil through apply()
  Attr2dgFn stream2dg_attr[kMaxTg + 1] = {};
  Occ2dgFn stream2dg_occ[kMaxTg + 1] = {};
  Stream1dLaunch stream1d[3] = {};  // [index of V in kStream1dVs]
  AttrFn stream1d_attr[3] = {};
};

// Programmatic dependent launch for the launches of a run (the kernels open
// with grid_dependency_sync()); OTS_PDL=0 in the environment turns it off.
inline bool launch_overlap() {
  static const bool on = [] {
    const char* v = std::getenv("OTS_PDL");
    return !(v && v[0] == '0');
  }();
  return on;
}

// cudaLaunchKernelEx with the dependent-launch attribute and, for cy > 1,
// thread-block clusters of cy CTAs along grid y.
template <class... Exp, class... Act>
cudaError_t launch_k(void (*kernel)(Exp...), dim3 g, dim3 b, size_t smem, cudaStream_t s,
                     int cy, Act&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  unsigned n = 0;
  if (launch_overlap() && cy <= 1) {  // clustered launches keep plain stream order
    attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  if (cy > 1) {
    attr[n].id = cudaLaunchAttributeClusterDimension;
    attr[n].val.clusterDim.x = 1;
    attr[n].val.clusterDim.y = (unsigned)cy;
    attr[n].val.clusterDim.z = 1;
    ++n;
  }
  cfg.attrs = attr;
  cfg.numAttrs = n;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...);
}

template <class K>
inline cudaError_t ensure_smem(K kernel, size_t smem, std::atomic<size_t>& cached) {
  if (smem <= 48 * 1024 || smem <= cached.load(std::memory_order_relaxed)) return cudaSuccess;
  cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) cached.store(smem, std::memory_order_relaxed);
  return e;
}

template <class Op, int E, int EAX>
cudaError_t launch_tile(const StepParams& p, dim3 g, dim3 b, size_t smem, cudaStream_t s) {
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(tile_kernel<Op, E, EAX>, smem, cached);
  if (e != cudaSuccess) return e;
  return launch_k(tile_kernel<Op, E, EAX>, g, b, smem, s, 1, p);
}

template <class Op, int E, int EAX>
cudaError_t attr_tile(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, tile_kernel<Op, E, EAX>);
}

template <class Op, int E>
cudaError_t launch_tex(const StepParams& p, dim3 g, dim3 b, size_t smem, cudaStream_t s) {
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(tile_tex_kernel<Op, E>, smem, cached);
  if (e != cudaSuccess) return e;
  return launch_k(tile_tex_kernel<Op, E>, g, b, smem, s, 1, p);
}

template <class Op, int E>
cudaError_t attr_tex(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, tile_tex_kernel<Op, E>);
}

template <class Op>
cudaError_t launch_plain(const StepParams& p, dim3 g, dim3 b, size_t, cudaStream_t s) {
  return launch_k(plain_kernel<Op>, g, b, 0, s, 1, p);
}

template <class Op>
cudaError_t attr_plain(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, plain_kernel<Op>);
}

template <class Op, int T, int E>
cudaError_t launch_stream(const CUtensorMap& m, const StreamParams& p, dim3 g, dim3 b,
                          size_t smem, cudaStream_t s) {
  if (p.cy > 1) {  // thread-block clusters of cy CTAs along grid y
    static std::atomic<size_t> cached_cl{0};
    cudaError_t e = ensure_smem(stream_kernel<Op, T, E, true>, smem, cached_cl);
    if (e != cudaSuccess) return e;
    return launch_k(stream_kernel<Op, T, E, true>, g, b, smem, s, p.cy, m, p);
  }
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(stream_kernel<Op, T, E, false>, smem, cached);
  if (e != cudaSuccess) return e;
  return launch_k(stream_kernel<Op, T, E, false>, g, b, smem, s, 1, m, p);
}

template <class Op, int T, int E>
cudaError_t attr_stream(cudaFuncAttributes* a, bool cl) {
  return cl ? cudaFuncGetAttributes(a, stream_kernel<Op, T, E, true>)
            : cudaFuncGetAttributes(a, stream_kernel<Op, T, E, false>);
}

template <class Op, int T, int E, bool CL>
cudaError_t occ_stream_k(int* blocks, int threads, size_t smem) {
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(stream_kernel<Op, T, E, CL>, smem, cached);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, stream_kernel<Op, T, E, CL>,
                                                       threads, smem);
}

template <class Op, int T, int E>
cudaError_t occ_stream(int* blocks, int threads, size_t smem, bool cl) {
  return cl ? occ_stream_k<Op, T, E, true>(blocks, threads, smem)
            : occ_stream_k<Op, T, E, false>(blocks, threads, smem);
}

template <class Op, int T, int SI>
cudaError_t launch_stream3p(const CUtensorMap& m, const StreamParams& p, dim3 g, dim3 b,
                            size_t smem, cudaStream_t s) {
  constexpr Shape3p S = kShape3p[SI];
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(stream3p_kernel<Op, T, S.E, S.BX, S.BY>, smem, cached);
  if (e != cudaSuccess) return e;
  return launch_k(stream3p_kernel<Op, T, S.E, S.BX, S.BY>, g, b, smem, s, 1, m, p);
}

template <class Op, int T, int SI>
cudaError_t attr_stream3p(cudaFuncAttributes* a) {
  constexpr Shape3p S = kShape3p[SI];
  return cudaFuncGetAttributes(a, stream3p_kernel<Op, T, S.E, S.BX, S.BY>);
}

template <class Op, int T, int SI>
cudaError_t occ_stream3p(int* blocks, int threads, size_t smem) {
  constexpr Shape3p S = kShape3p[SI];
  static std::atomic<size_t> cached{0};
  cudaError_t e = ensure_smem(stream3p_kernel<Op, T, S.E, S.BX, S.BY>, smem, cached);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      blocks, stream3p_kernel<Op, T, S.E, S.BX, S.BY>, threads, smem);
}

// One shape of the packed kernel for every T (compiled where it is called,
// one translation unit per shape group).
template <class Op, int SI, int... Ts>
void fill_stream3p_shape(StencilKernels& k, std::integer_sequence<int, Ts...>) {
  ((k.stream3p[Ts + 1][SI] = &launch_stream3p<Op, Ts + 1, SI>,
    k.stream3p_attr[Ts + 1][SI] = &attr_stream3p<Op, Ts + 1, SI>,
    k.stream3p_occ[Ts + 1][SI] = &occ_stream3p<Op, Ts + 1, SI>),
   ...);
}

// Defined in ots_k_{jacobi,poisson}_3d_p<N>.cu: the packed kernel's table
// entries.
void fill_stream3p_jacobi_3d_a(StencilKernels& k);
void fill_stream3p_jacobi_3d_b(StencilKernels& k);
void fill_stream3p_poisson_3d_a(StencilKernels& k);
void fill_stream3p_poisson_3d_b(StencilKernels& k);

template <class Op, int EAX, int... Es>
void fill_tile(StencilKernels& k, std::integer_sequence<int, Es...>) {
  ((k.tile[EAX][Es + 1] = &launch_tile<Op, Es + 1, EAX>,
    k.tile_attr[EAX][Es + 1] = &attr_tile<Op, Es + 1, EAX>),
   ...);
}

template <class Op, int T>
cudaError_t launch_stream2d(const Stream2dParams& p, dim3 g, cudaStream_t s) {
  return launch_k(stream2d_kernel<Op, T>, g, dim3(kStream2dThreads), 0, s, 1, p);
}

template <class Op, int T>
cudaError_t attr_stream2d(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, stream2d_kernel<Op, T>);
}

template <class Op, int T>
cudaError_t occ_stream2d(int* blocks) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, stream2d_kernel<Op, T>,
                                                       kStream2dThreads, 0);
}

template <class Op, int T>
cudaError_t launch_stream2dp(const Stream2dParams& p, dim3 g, cudaStream_t s) {
  return launch_k(stream2dp_kernel<Op, T>, g, dim3(kStream2dThreads), 0, s, 1, p);
}

template <class Op, int T>
cudaError_t attr_stream2dp(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, stream2dp_kernel<Op, T>);
}

template <class Op, int T>
cudaError_t occ_stream2dp(int* blocks) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, stream2dp_kernel<Op, T>,
                                                       kStream2dThreads, 0);
}

template <class Op, int V>
cudaError_t launch_stream1d(const Stream1dParams& p, dim3 g, cudaStream_t s) {
  return launch_k(stream1d_kernel<Op, V>, g, dim3(kStream1dThreads), 0, s, 1, p);
}

template <class Op, int V>
cudaError_t attr_stream1d(cudaFuncAttributes* a) {
  return cudaFuncGetAttributes(a, stream1d_kernel<Op, V>);
}

// The y-streamed kernel of a stencil without the five-point form: FDTD-2D
// and Rician-denoise-2D have their own two-phase kernels (Rician's in two
// instantiations, IEEE and fast division: `fast` picks one); every other op
// goes through its apply().
template <class Op, int T>
auto stream2dg_entry(bool fast = false) {
  (void)fast;
  if constexpr (std::is_same_v<Op, OpFdtd2D>)
    return &stream2d_fdtd_kernel<T>;
  else if constexpr (std::is_same_v<Op, OpRician2D>)
    return fast ? &stream2d_rician_kernel<T, true> : &stream2d_rician_kernel<T, false>;
  else
    return &stream2dg_kernel<Op, T>;
}

template <class Op, int T>
cudaError_t launch_stream2dg(const Stream2dgParams& p, dim3 g, cudaStream_t s) {
  return launch_k(stream2dg_entry<Op, T>(p.op.variant == 2), g, dim3(kStream2dThreads), 0, s, 1,
                  p);
}

template <class Op, int T>
cudaError_t attr_stream2dg(cudaFuncAttributes* a, bool fast) {
  return cudaFuncGetAttributes(a, stream2dg_entry<Op, T>(fast));
}

template <class Op, int T>
cudaError_t occ_stream2dg(int* blocks, bool fast) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, stream2dg_entry<Op, T>(fast),
                                                       kStream2dThreads, 0);
}

template <class Op, int... Ts>
void fill_stream2dg(StencilKernels& k, std::integer_sequence<int, Ts...>) {
  ((k.stream2dg[Ts + 1] = &launch_stream2dg<Op, Ts + 1>,
    k.stream2dg_attr[Ts + 1] = &attr_stream2dg<Op, Ts + 1>,
    k.stream2dg_occ[Ts + 1] = &occ_stream2dg<Op, Ts + 1>),
   ...);
}

template <class Op, int... Ts>
void fill_stream2dp(StencilKernels& k, std::integer_sequence<int, Ts...>) {
  ((k.stream2dp[Ts + 1] = &launch_stream2dp<Op, Ts + 1>,
    k.stream2dp_attr[Ts + 1] = &attr_stream2dp<Op, Ts + 1>,
    k.stream2dp_occ[Ts + 1] = &occ_stream2dp<Op, Ts + 1>),
   ...);
}

template <class Op, int... Ts>
void fill_stream2d(StencilKernels& k, std::integer_sequence<int, Ts...>) {
  ((k.stream2d[Ts + 1] = &launch_stream2d<Op, Ts + 1>,
    k.stream2d_attr[Ts + 1] = &attr_stream2d<Op, Ts + 1>,
    k.stream2d_occ[Ts + 1] = &occ_stream2d<Op, Ts + 1>),
   ...);
}

template <class Op, int... Es>
void fill_tex(StencilKernels& k, std::integer_sequence<int, Es...>) {
  ((k.tex[Es + 1] = &launch_tex<Op, Es + 1>, k.tex_attr[Es + 1] = &attr_tex<Op, Es + 1>), ...);
}

template <class Op, int EI, int... Ts>
void fill_stream_e(StencilKernels& k, std::integer_sequence<int, Ts...>) {
  ((k.stream[Ts + 1][EI] = &launch_stream<Op, Ts + 1, kStreamEs[EI]>,
    k.stream_attr[Ts + 1][EI] = &attr_stream<Op, Ts + 1, kStreamEs[EI]>,
    k.stream_occ[Ts + 1][EI] = &occ_stream<Op, Ts + 1, kStreamEs[EI]>),
   ...);
}

template <class Op>
StencilKernels make_kernels() {
  StencilKernels k;
  if constexpr (Op::DIMS == 1) {
    fill_tile<Op, 0>(k, std::make_integer_sequence<int, kMaxE>{});
    k.stream1d[0] = &launch_stream1d<Op, 4>;
    k.stream1d[1] = &launch_stream1d<Op, 8>;
    k.stream1d[2] = &launch_stream1d<Op, 16>;
    k.stream1d_attr[0] = &attr_stream1d<Op, 4>;
    k.stream1d_attr[1] = &attr_stream1d<Op, 8>;
    k.stream1d_attr[2] = &attr_stream1d<Op, 16>;
  }
  if constexpr (Op::DIMS == 2) fill_tile<Op, 1>(k, std::make_integer_sequence<int, kMaxE>{});
  if constexpr (Op::DIMS == 2 && Op::NS == 1)
    fill_tex<Op>(k, std::make_integer_sequence<int, kTexMaxE>{});
  if constexpr (Op::DIMS == 2 && HasStar2D<Op>::value)
    fill_stream2d<Op>(k, std::make_integer_sequence<int, kMaxT>{});
  if constexpr (Op::DIMS == 2 && Packed2D<Op>::value)
    fill_stream2dp<Op>(k, std::make_integer_sequence<int, kMaxT>{});
  // the generic streamed kernel where the five-point form does not cover the
  // op (several fields, aux fields, or other neighbours)
  if constexpr (Op::DIMS == 2 && (Op::NS > 1 || Op::NA > 0 || !HasStar2D<Op>::value))
    fill_stream2dg<Op>(k, std::make_integer_sequence<int, kMaxTg>{});
  if constexpr (Op::DIMS == 3) {
    fill_tile<Op, 2>(k, std::make_integer_sequence<int, kMaxE3>{});
    fill_tile<Op, 1>(k, std::make_integer_sequence<int, kMaxE3>{});
  }
  k.plain = &launch_plain<Op>;
  k.plain_attr = &attr_plain<Op>;
  return k;
}

template <class Op>
StencilKernels make_kernels_with_stream() {
  StencilKernels k = make_kernels<Op>();
  fill_stream_e<Op, 0>(k, std::make_integer_sequence<int, kMaxT>{});
  fill_stream_e<Op, 1>(k, std::make_integer_sequence<int, kMaxT>{});
  fill_stream_e<Op, 2>(k, std::make_integer_sequence<int, kMaxT>{});
  k.has_stream = true;
  return k;
}

// Defined one per stencil in ots_k_<stencil>.cu.
const StencilKernels& kernels_for(int stencil);

}  // namespace ots
