// ref_clkernel.cpp -- runs ONE kernel text emitted by the reference's own
// generator (XGenerator::generate) on the CPU, for pinning the oracle.
//
// TEST INFRASTRUCTURE ONLY (the checker, never the product).  The reference
// runners build their kernels with OpenCL, which is absent here; the kernel
// text itself is plain OpenCL C that also parses as C++ once the few OpenCL
// words it uses are given meanings.  oracle/build_ref.py writes the text for
// one (stencil, problem size, block, T, E) case to oracle/_ref/ and compiles
// this file with -DOTS_CL_KERNEL_FILE="<that file>" -DOTS_CL_STENCIL=<id>
// into one shared library per case (git-ignored, never committed).
//
// Work-item model (OpenCL 1.x execution semantics):
//   * one std::thread per work-item of a work-group; the work-groups of a
//     launch run one after another, in group-id order;
//   * barrier() is a std::barrier over the group's work-items;
//   * __local arrays are function-scope statics, shared by the group's
//     work-items; they start zeroed and a slot that no work-item writes keeps
//     its zero (the generated kernels read such slots only at a tile edge,
//     where a tile that covers the whole interior reads the zero ring);
//   * get_local_id / get_group_id / get_local_size / get_num_groups return
//     size_t as in OpenCL.
// Maths: rsqrt(x) = 1.0f / sqrtf(x) for float and 1.0 / sqrt(x) for double
// arguments, pow(x, 2.0f) = x * x (the correctly rounded values; the CPU
// oracle evaluates them the same way), and
// the file is compiled with -ffp-contract=off so every operation of the text
// is its own IEEE single operation.
//
// Launch loops follow each runner's main(): ceil(S/T) launches with the
// baseTime argument and in/out swapped after each (e.g.
// opencl/jacobi-3d/jacobi-3d.cpp:789-818), floor(S/T) launches without it for
// cs-3d (opencl/cs-3d/cs-3d.cpp:764-779); NDRange = numBlocks x blockSize per
// dimension (opencl/jacobi-3d/jacobi-3d.cpp:769-774); the result is the
// final input buffer (:834).
#include <barrier>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace clemu {
thread_local size_t lid[3], gid[3];
size_t lsz[3] = {1, 1, 1}, ngr[3] = {1, 1, 1};
std::barrier<>* bar = nullptr;
}  // namespace clemu

static inline size_t get_local_id(int d) { return clemu::lid[d]; }
static inline size_t get_group_id(int d) { return clemu::gid[d]; }
static inline size_t get_local_size(int d) { return clemu::lsz[d]; }
static inline size_t get_num_groups(int d) { return clemu::ngr[d]; }
static inline void barrier(int) { clemu::bar->arrive_and_wait(); }
static inline float ots_cl_rsqrt(float v) { return 1.0f / sqrtf(v); }
static inline double ots_cl_rsqrt(double v) { return 1.0 / sqrt(v); }
static inline float ots_cl_pow(float a, float b) { return b == 2.0f ? a * a : powf(a, b); }

#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
#define __kernel
#define __global
#define __local static
#define rsqrt(v) ots_cl_rsqrt(v)
#define pow(a, b) ots_cl_pow((a), (b))

#include OTS_CL_KERNEL_FILE

#undef pow
#undef rsqrt
#undef __local

namespace {

// One launch: every work-group in order, each run by its own work-items.
template <class F>
void launch(const int nb[3], const int bs[3], F&& body) {
  for (int d = 0; d < 3; ++d) {
    clemu::lsz[d] = (size_t)bs[d];
    clemu::ngr[d] = (size_t)nb[d];
  }
  const int W = bs[0] * bs[1] * bs[2];
  for (int g2 = 0; g2 < nb[2]; ++g2)
    for (int g1 = 0; g1 < nb[1]; ++g1)
      for (int g0 = 0; g0 < nb[0]; ++g0) {
        std::barrier<> b(W);
        clemu::bar = &b;
        std::vector<std::thread> th;
        th.reserve(W);
        for (int w = 0; w < W; ++w)
          th.emplace_back([=, &body]() {
            clemu::gid[0] = (size_t)g0;
            clemu::gid[1] = (size_t)g1;
            clemu::gid[2] = (size_t)g2;
            clemu::lid[0] = (size_t)(w % bs[0]);
            clemu::lid[1] = (size_t)((w / bs[0]) % bs[1]);
            clemu::lid[2] = (size_t)(w / (bs[0] * bs[1]));
            body();
          });
        for (auto& t : th) t.join();
        clemu::bar = nullptr;
      }
}

}  // namespace

// fields: the evolving arrays (P^dims floats each, reference layout), run in
// place; aux: read-only arrays in the runner's argument order; nb/bs: the
// runner's numBlocks and blockSize per dimension (1 for unused dimensions).
extern "C" int clk_run(float** fields, float** aux, int nfields, int P, int dims, int T,
                       int steps, const int* nb, const int* bs) {
  size_t cells = 1;
  for (int d = 0; d < dims; ++d) cells *= (size_t)P;
  // the runners write the input to both device buffers
  // (opencl/jacobi-3d/jacobi-3d.cpp:746-753)
  std::vector<std::vector<float>> A(nfields), B(nfields);
  for (int f = 0; f < nfields; ++f) {
    A[f].assign(fields[f], fields[f] + cells);
    B[f] = A[f];
  }
  std::vector<float*> in(nfields), out(nfields);
  for (int f = 0; f < nfields; ++f) {
    in[f] = A[f].data();
    out[f] = B[f].data();
  }
#if OTS_CL_STENCIL == 12
  const int launches = steps / T;  // cs-3d: floor(S/T), no baseTime
#else
  const int launches = (steps + T - 1) / T;
#endif
  for (int l = 0; l < launches; ++l) {
    const unsigned t = (unsigned)(l * T);
    (void)t;
#if OTS_CL_STENCIL == 9  // fdtd-2d: (EX, EY, HZ in; EX, EY, HZ out; t)
    launch(nb, bs, [&]() { kernel_func(in[0], in[1], in[2], out[0], out[1], out[2], t); });
#elif OTS_CL_STENCIL == 10  // rician-denoise-2d: (input, F, output, t)
    launch(nb, bs, [&]() { kernel_func(in[0], aux[0], out[0], t); });
#elif OTS_CL_STENCIL == 11  // cdsc-tv-update-2d: (input, V, F, output, t)
    launch(nb, bs, [&]() { kernel_func(in[0], aux[0], aux[1], out[0], t); });
#elif OTS_CL_STENCIL == 12  // cs-3d: (input, output)
    launch(nb, bs, [&]() { kernel_func(in[0], out[0]); });
#else  // jacobi-3d, poisson-3d, gradient-3d: (input, output, t)
    launch(nb, bs, [&]() { kernel_func(in[0], out[0], t); });
#endif
    std::swap(in, out);
  }
  for (int f = 0; f < nfields; ++f) std::memcpy(fields[f], in[f], cells * sizeof(float));
  return 0;
}
