// ots_runtime.cu -- the C ABI of include/ots.h.
//
// Replaces the reference's opencl/common library (CLContext, throwOnError,
// ProgramGenerator::printProgramParameters, rtclock/printValue) and the
// per-stencil runner main()s (e.g. opencl/jacobi-2d/jacobi-2d.cpp:553-1048):
// geometry derivation, device buffers, uploads, the launch loop with event
// timing, read-back and the key/value report, for one B200.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/ots.h"
#include "ots_launch.cuh"

namespace ots {
const StencilKernels& kernels_jacobi_1d();
const StencilKernels& kernels_jacobi_1d_5pt();
const StencilKernels& kernels_jacobi_1d_7pt();
const StencilKernels& kernels_jacobi_2d();
const StencilKernels& kernels_jacobi_3d();
const StencilKernels& kernels_poisson_2d();
const StencilKernels& kernels_poisson_3d();
const StencilKernels& kernels_gradient_2d();
const StencilKernels& kernels_gradient_3d();
const StencilKernels& kernels_fdtd_2d();
const StencilKernels& kernels_rician_denoise_2d();
const StencilKernels& kernels_cdsc_tv_update_2d();
const StencilKernels& kernels_cs_3d();

const StencilKernels& kernels_for(int s) {
  switch (s) {
    case OTS_JACOBI_1D: return kernels_jacobi_1d();
    case OTS_JACOBI_1D_5PT: return kernels_jacobi_1d_5pt();
    case OTS_JACOBI_1D_7PT: return kernels_jacobi_1d_7pt();
    case OTS_JACOBI_2D: return kernels_jacobi_2d();
    case OTS_JACOBI_3D: return kernels_jacobi_3d();
    case OTS_POISSON_2D: return kernels_poisson_2d();
    case OTS_POISSON_3D: return kernels_poisson_3d();
    case OTS_GRADIENT_2D: return kernels_gradient_2d();
    case OTS_GRADIENT_3D: return kernels_gradient_3d();
    case OTS_FDTD_2D: return kernels_fdtd_2d();
    case OTS_RICIAN_DENOISE_2D: return kernels_rician_denoise_2d();
    case OTS_CDSC_TV_UPDATE_2D: return kernels_cdsc_tv_update_2d();
    default: return kernels_cs_3d();
  }
}
}  // namespace ots

namespace {

// ------------------------------------------------------------ metadata --

struct StencilInfo {
  const char* name;
  int dims, ns, na;
  int rx, ry, rz;    // per-step dependence radius of the fused update
  int ref_r;         // radius the reference geometry uses (padding = ref_r*T)
  bool star;         // 7-point star form available (stream kernel)
  double flops;      // reference "Actual GFlop/s" constant per point
  // printProgramParameters arguments where the runner passes them
  // (numArrays, loads/pt, stores/pt, flops/pt); 0 = runner prints none.
  int pp_arrays, pp_loads, pp_stores, pp_flops;
  // model constants the runner prints (phase2_global_loads ...); -1 = none
  double r5[8];
  // the tile step runs in two phases with one float per tile cell of phase-1
  // values in shared memory (the op's TWO_PHASE form)
  bool two_phase = false;
};

// flops: opencl/<s>/<s>.cpp "double gflops" lines (jacobi-2d.cpp:1001-1002,
// jacobi-3d.cpp:915-917, poisson-2d.cpp:746-747, poisson-3d.cpp:881-883,
// gradient-2d.cpp:797-798, gradient-3d.cpp:917-919, fdtd-2d.cpp:885-886,
// rician-denoise-2d.cpp:844, cdsc-tv-update-2d.cpp:569, cs-3d.cpp:796-798,
// jacobi-1d.cpp:808-809, jacobi-1d-5pt.cpp:588-589, jacobi-1d-7pt.cpp:598-599).
// r5: jacobi-2d.cpp:1029-1036 and the matching lines of each runner.
const StencilInfo kInfo[OTS_NUM_STENCILS] = {
    {"jacobi-1d", 1, 1, 0, 1, 0, 0, 1, false, 3, 1, 3, 1, 3, {3, 0, 3, 3, 1, 1, 1, 4}},
    {"jacobi-1d-5pt", 1, 1, 0, 2, 0, 0, 2, false, 5, 0, 0, 0, 0, {-1}},
    {"jacobi-1d-7pt", 1, 1, 0, 3, 0, 0, 3, false, 7, 0, 0, 0, 0, {-1}},
    {"jacobi-2d", 2, 1, 0, 1, 1, 0, 1, true, 5, 1, 5, 1, 5, {5, 0, 5, 5, 1, 1, 1, 4}},
    {"jacobi-3d", 3, 1, 0, 1, 1, 1, 1, true, 7, 0, 0, 0, 0, {7, 0, 7, 5, 1, 1, 1, 4}},
    {"poisson-2d", 2, 1, 1, 1, 1, 0, 1, false, 9, 1, 9, 1, 9, {9, 0, 9, 9, 1, 1, 1, 4}},
    {"poisson-3d", 3, 1, 1, 1, 1, 1, 1, true, 27, 0, 0, 0, 0, {27, 0, 27, 27, 1, 1, 1, 4}},
    {"gradient-2d", 2, 1, 0, 1, 1, 0, 1, true, 15, 1, 5, 1, 18, {5, 0, 12, 5, 1, 1, 1, 4}},
    {"gradient-3d", 3, 1, 0, 1, 1, 1, 1, true, 20, 0, 0, 0, 0, {7, 0, 20, 7, 1, 1, 1, 4}},
    {"fdtd-2d", 2, 3, 0, 1, 1, 0, 1, false, 11, 3, 8, 3, 11, {7, 4, 11, 5, 3, 3, 3, 4}},
    {"rician-denoise-2d", 2, 1, 1, 2, 2, 0, 1, false, 42, 3, 6, 3, 44, {13, 0, 42, 13, 1, 1, 1, 4},
     true},
    {"cdsc-tv-update-2d", 2, 1, 2, 1, 1, 0, 1, false, 59, 1, 7, 1, 59, {7, 0, 59, 7, 1, 1, 1, 4}},
    {"cs-3d", 3, 1, 0, 1, 1, 1, 1, false, 65, 0, 0, 0, 0, {-1}},
};

thread_local std::string g_last_error;
}  // namespace

void ots_set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

namespace {

ots_status fail(ots_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

ots_status cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation)
    return fail(OTS_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
  return fail(OTS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define OTS_CUDA(call, what)                          \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

int gcd_i(int a, int b) {
  a = a < 0 ? -a : a;
  b = b < 0 ? -b : b;
  while (b) {
    int t = a % b;
    a = b;
    b = t;
  }
  return a;
}
int lcm_i(int a, int b) {
  if (a == 0 || b == 0) return 0;
  int l = a / gcd_i(a, b) * b;
  return l < 0 ? -l : l;
}
int ceil_div(int a, int b) { return (a + b - 1) / b; }
int64_t round_up(int64_t a, int64_t m) { return (a + m - 1) / m * m; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// 1D register kernel: warps of 32 x V cells, T steps in registers
struct Stream1dCfg {
  int V = 0, vidx = 0, hx = 0, rpb = 0, nw = 0, grid = 0;
};

// y-streamed 2D kernel: 128-cell strips x y segments, one warp each
struct Stream2dCfg {
  int T = 0, hx = 0, rpbx = 0, ntx = 0, nseg = 0, zseg = 0, grid = 0;
  int warps_per_sm = 0;
  bool generic = false;  // stream2dg_kernel (the op's apply through register rows)
  bool packed = false;   // stream2dp_kernel (packed FP32 five-point form)
  int R = 1;             // rows of reach per level
};

struct StreamCfg {
  int T = 0, E = 0, eidx = 0, bx = 0, by = 0;
  bool packed = false;     // the packed-FP32 kernel (ots_stream3p.cuh)
  int shape3p = -1;        // its block shape (index in kShape3p)
  int cy = 1;              // CTAs per cluster along y (their tiles stack into one)
  int tx = 0, ty = 0, rpbx = 0, rpby = 0, zseg = 0;
  int nbx = 0, nby = 0, nbz = 0;
  int grid = 0;            // persistent CTAs launched
  int64_t work = 0;        // output tile-planes
  int64_t chunk = 0;       // tile-planes per CTA
  size_t smem = 0;
};

}  // namespace

struct ots_plan {
  ots_params prm{};
  ots_geometry geo{};
  const StencilInfo* info = nullptr;
  const ots::StencilKernels* K = nullptr;
  int device = 0;
  int sm_count = 0;
  size_t smem_optin = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ots::Layout L{};
  int64_t field_elems = 0;
  float* state[2][3] = {};
  float* aux[2] = {};
  int cur = 0;
  int* d_err = nullptr;
  uint64_t wait_ns = ots::kWaitNs;  // limit of the stream kernel's bounded waits
  int hold_plane = -1;              // test hook (ots_plan_debug_hold_plane)
  // -c clock recording (tile kernel): kClockWords per warp of the last launch
  unsigned* d_clocks = nullptr;
  int64_t clock_warps = 0;
  bool clocks_valid = false;  // the last run used the tile kernel
  ots::OpArgs op{};
  CUtensorMap tmap[2];  // stream kernel: field 0 of state buffer 0 / 1
  CUtensorMap amap;     // stream kernel: aux field 0 (Poisson f), same box
  bool tmap_ok = false;
  cudaTextureObject_t tex[2] = {0, 0};  // texture kernel: field 0 of state buffer 0 / 1
  bool tex_ok = false;
  StreamCfg scfg;
  Stream2dCfg s2cfg;
  Stream1dCfg s1cfg;
  // tile kernel launch shape
  dim3 tile_grid, tile_block;
  size_t tile_smem = 0;
  int eaxis = 1;
};

namespace {

// ------------------------------------------------------------- geometry --

ots_status derive(const ots_params* p, ots_geometry* g, const StencilInfo** info_out) {
  if (!p) return fail(OTS_ERR_INVALID_ARGUMENT, "params is NULL");
  if (p->stencil < 0 || p->stencil >= OTS_NUM_STENCILS)
    return fail(OTS_ERR_INVALID_ARGUMENT, "unknown stencil id %d", p->stencil);
  for (int i = 0; i < 5; ++i)
    if (p->reserved[i] != 0) return fail(OTS_ERR_INVALID_ARGUMENT, "reserved fields must be 0");
  if (p->stream_impl < 0 || p->stream_impl > 1)
    return fail(OTS_ERR_INVALID_ARGUMENT, "stream_impl must be 0 or 1 (got %d)", p->stream_impl);
  if (p->cluster_y < 0 || p->cluster_y > 8)
    return fail(OTS_ERR_INVALID_ARGUMENT, "cluster_y must be 0..8 (got %d)", p->cluster_y);
  const StencilInfo& si = kInfo[p->stencil];
  if (info_out) *info_out = &si;
  const int d = si.dims;
  const int n = p->problem_size, T = p->time_tile, E = p->elements_per_thread;
  const int bx = p->block_x, by = d >= 2 ? p->block_y : 1, bz = d == 3 ? p->block_z : 1;
  if (n < 1) return fail(OTS_ERR_INVALID_ARGUMENT, "problem size must be >= 1 (got %d)", n);
  if (p->time_steps < 0) return fail(OTS_ERR_INVALID_ARGUMENT, "time steps must be >= 0");
  if (T < 1) return fail(OTS_ERR_INVALID_ARGUMENT, "time tile size must be >= 1 (got %d)", T);
  if (E < 1) return fail(OTS_ERR_INVALID_ARGUMENT, "elements per thread must be >= 1");
  if (bx < 1 || by < 1 || bz < 1) return fail(OTS_ERR_INVALID_ARGUMENT, "block sizes must be >= 1");
  if (p->engine != OTS_ENGINE_NATIVE && p->engine != OTS_ENGINE_COMPAT)
    return fail(OTS_ERR_INVALID_ARGUMENT, "unknown engine %d", p->engine);
  if (p->kernel < OTS_KERNEL_AUTO || p->kernel > OTS_KERNEL_TEX)
    return fail(OTS_ERR_INVALID_ARGUMENT, "unknown kernel family %d", p->kernel);
  if (p->variant != OTS_VARIANT_BASELINE && p->variant != OTS_VARIANT_REF &&
      p->variant != OTS_VARIANT_FAST)
    return fail(OTS_ERR_INVALID_ARGUMENT, "unknown variant %d", p->variant);
  if (p->variant == OTS_VARIANT_FAST && p->stencil != OTS_RICIAN_DENOISE_2D &&
      p->stencil != OTS_CDSC_TV_UPDATE_2D && p->stencil != OTS_CS_3D)
    return fail(OTS_ERR_INVALID_ARGUMENT,
                "the fast-division variant applies to rician-denoise-2d, cdsc-tv-update-2d "
                "and cs-3d only");
  if (p->phase_limit < 0 || p->phase_limit > 3)
    return fail(OTS_ERR_INVALID_ARGUMENT, "phase limit must be 0..3");

  memset(g, 0, sizeof(*g));
  g->dims = d;
  g->radius = std::max(si.rx, std::max(si.ry, si.rz));
  g->num_fields = si.ns;
  g->num_aux = si.na;
  g->flops_per_point = si.flops;
  g->e_axis = d == 1 ? 0 : (d == 2 ? 1 : (p->engine == OTS_ENGINE_COMPAT ? 1 : 2));

  // Reference derivation (GeneratorParams::computeDerived):
  //   1D  opencl/jacobi-1d/jacobi-1d.cpp:75-105 (+109 pad), jacobi-1d-5pt.cpp:59-86
  //   2D  opencl/jacobi-2d/jacobi-2d.cpp:84-126 (gcd), poisson-2d.cpp:80 (lcm)
  //   3D  opencl/jacobi-3d/jacobi-3d.cpp:78-114 (lcm, E on y)
  int comps[3] = {1, 1, 1}, rrpb[3] = {1, 1, 1};
  const int rr = si.ref_r;
  if (d == 1) {
    comps[0] = bx * E;
    rrpb[0] = comps[0] - 2 * rr * (T - 1);
  } else {
    comps[0] = bx;
    comps[1] = by * E;
    comps[2] = d == 3 ? bz : 1;
    rrpb[0] = comps[0] - 2 * (T - 1);
    rrpb[1] = comps[1] - 2 * (T - 1);
    rrpb[2] = d == 3 ? comps[2] - 2 * (T - 1) : 1;
  }
  int size_lcm;
  if (d == 1) size_lcm = rrpb[0];
  else if (d == 2)
    size_lcm = p->stencil == OTS_POISSON_2D ? lcm_i(rrpb[0], rrpb[1]) : gcd_i(rrpb[0], rrpb[1]);
  else
    size_lcm = lcm_i(rrpb[2], lcm_i(rrpb[0], rrpb[1]));
  g->shared_size[0] = d == 1 ? bx * E + 2 * rr : bx + 2;
  g->shared_size[1] = d >= 2 ? by * E + 2 : 1;
  g->shared_size[2] = d == 3 ? bz + 2 : 1;

  if (p->engine == OTS_ENGINE_COMPAT) {
    if (rrpb[0] < 1 || rrpb[1] < 1 || rrpb[2] < 1 || size_lcm < 1)
      return fail(OTS_ERR_INVALID_GEOMETRY,
                  "Consistency error! real per block (%d, %d, %d) must be >= 1", rrpb[0],
                  rrpb[1], rrpb[2]);
    g->size_lcm = size_lcm;
    g->real_size = (n / size_lcm) * size_lcm;
    if (g->real_size < 1)
      return fail(OTS_ERR_INVALID_GEOMETRY,
                  "Consistency error! problem size %d truncates to 0 (sizeLCM %d)", n, size_lcm);
    for (int a = 0; a < d; ++a)
      if (g->real_size / rrpb[a] < 1)
        return fail(OTS_ERR_INVALID_GEOMETRY,
                    "Consistency error! no whole block fits along axis %d (real size %d, real "
                    "per block %d)",
                    a, g->real_size, rrpb[a]);
    g->padding = rr * T;
    g->padded_size = g->real_size + 2 * g->padding + (p->stencil == OTS_JACOBI_1D ? 109 : 0);
  } else {
    g->size_lcm = size_lcm > 0 ? size_lcm : 1;
    g->real_size = n;
    g->padding = rr * T;
    g->padded_size = n + 2 * g->padding;
  }
  g->interior_points = 1;
  for (int a = 0; a < d; ++a) g->interior_points *= g->real_size;
  g->launches = p->time_steps > 0 ? ceil_div(p->time_steps, T) : 0;

  // Tile-kernel geometry with the true radius and the engine's E axis.
  const int R[3] = {si.rx, si.ry, si.rz};
  int tc[3] = {bx, by, bz};
  tc[g->e_axis] *= E;
  for (int a = 0; a < 3; ++a) {
    g->comps[a] = a < d ? tc[a] : 1;
    g->real_per_block[a] = a < d ? tc[a] - 2 * R[a] * (T - 1) : 1;
    g->num_blocks[a] = a < d ? (g->real_per_block[a] >= 1
                                    ? ceil_div(g->real_size, g->real_per_block[a])
                                    : 0)
                             : 1;
  }
  g->threads[0] = bx;
  g->threads[1] = by;
  g->threads[2] = bz;
  int64_t useful = 1, total = 1;
  for (int a = 0; a < d; ++a) {
    useful *= std::max(0, g->real_per_block[a]);
    total *= g->comps[a];
  }
  g->useful_ratio = total > 0 ? (double)useful / (double)total : 0.0;
  return OTS_OK;
}

// 2D stream kernel: strips of 128 cells along x (x halo T rounded up to 4 per side), rows split
// into segments (block_y > 1: that many rows per segment; else
// stream2d_zseg's choice).
// 1D: E = cells per lane (4, 8 or 16); the strip keeps 32 E - 2 roundup4(R T)
// output cells (multiple of 4); the same strips serve shallower launches.
ots_status derive_stream1d(const ots_plan* pl, Stream1dCfg* c) {
  const ots_params& p = pl->prm;
  c->vidx = -1;
  for (int i = 0; i < 3; ++i)
    if (ots::kStream1dVs[i] == p.elements_per_thread) c->vidx = i;
  if (c->vidx < 0 || !pl->K || !pl->K->stream1d[c->vidx])
    return fail(OTS_ERR_UNSUPPORTED, "1D stream kernel supports E in {4, 8, 16} (got %d)",
                p.elements_per_thread);
  c->V = p.elements_per_thread;
  c->rpb = ots::stream1d_rpb(c->V, pl->info->rx, p.time_tile, &c->hx);
  if (c->rpb < 4)
    return fail(OTS_ERR_INVALID_GEOMETRY,
                "Consistency error! a warp of %d cells leaves no interior at T=%d", 32 * c->V,
                p.time_tile);
  c->nw = ceil_div(pl->geo.real_size, c->rpb);
  const int wpc = ots::kStream1dThreads / 32;
  c->grid = ceil_div(c->nw, wpc);
  return OTS_OK;
}

bool star2d_usable(const ots_plan* pl) {
  return pl->K && pl->K->stream2d[1] &&
         !(pl->prm.stencil == OTS_POISSON_2D && pl->prm.variant == OTS_VARIANT_REF);
}

ots_status derive_stream2d(const ots_plan* pl, int T, Stream2dCfg* c) {
  c->generic = !star2d_usable(pl);
  c->R = c->generic ? pl->info->ry : 1;
  const int maxT = c->generic ? ots::kMaxTg : ots::kMaxT;
  const bool have = T >= 1 && T <= maxT && pl->K &&
                    (c->generic ? pl->K->stream2dg[T] != nullptr : pl->K->stream2d[T] != nullptr);
  if (!have)
    return fail(OTS_ERR_UNSUPPORTED, "2D stream kernel supports T in 1..%d (got %d)", maxT, T);
  c->T = T;
  c->hx = ots::stream2d_halo(c->R * T);
  c->rpbx = ots::kStream2dWidth - 2 * c->hx;
  const int n = pl->geo.real_size;
  c->ntx = ceil_div(n, c->rpbx);
  // the packed form where the op has one (any row width); stream_impl 1
  // keeps the scalar kernel
  c->packed = !c->generic && pl->prm.stream_impl != 1 && pl->K->stream2dp[T] != nullptr;
  int blocks = 0;
  const bool fast = pl->prm.variant == OTS_VARIANT_FAST;
  cudaError_t oe = cudaErrorInvalidValue;
  if (c->generic && pl->K->stream2dg_occ[T])
    oe = pl->K->stream2dg_occ[T](&blocks, fast);
  else if (c->packed && pl->K->stream2dp_occ[T])
    oe = pl->K->stream2dp_occ[T](&blocks);
  else if (!c->generic && pl->K->stream2d_occ[T])
    oe = pl->K->stream2d_occ[T](&blocks);
  if (oe != cudaSuccess || blocks < 1) blocks = 1;
  c->warps_per_sm = blocks * (ots::kStream2dThreads / 32);
  c->zseg = ots::stream2d_zseg(n, c->R * T, c->ntx, pl->sm_count, c->warps_per_sm);
  // block_y > 1 sets the rows per segment directly (tuning); else the model
  if (pl->prm.block_y > 1) c->zseg = std::min(n, pl->prm.block_y);
  c->nseg = ceil_div(n, c->zseg);
  const int64_t warps = (int64_t)c->ntx * c->nseg;
  c->grid = (int)((warps + ots::kStream2dThreads / 32 - 1) / (ots::kStream2dThreads / 32));
  return OTS_OK;
}

// Stream-kernel shape: bx threads x 4 cells along x, by threads x E rows
// along y; z split into segments so the CTA count fills whole waves.
ots_status derive_stream(const ots_plan* pl, int T, StreamCfg* c) {
  const ots_params& p = pl->prm;
  int eidx = -1;
  for (int i = 0; i < 3; ++i)
    if (ots::kStreamEs[i] == p.elements_per_thread) eidx = i;
  if (eidx < 0)
    return fail(OTS_ERR_UNSUPPORTED, "stream kernel supports E in {1, 2, 4} (got %d)",
                p.elements_per_thread);
  if (T < 1 || T > ots::kMaxT)
    return fail(OTS_ERR_UNSUPPORTED, "stream kernel supports T in 1..%d (got %d)", ots::kMaxT, T);
  c->T = T;
  c->E = p.elements_per_thread;
  c->eidx = eidx;
  c->bx = p.block_x;
  c->by = p.block_y;
  const int hx = (T + 3) / 4 * 4, hy = T;
  c->cy = p.cluster_y > 1 ? p.cluster_y : 1;
  c->tx = 4 * c->bx;
  c->ty = c->E * c->by;
  c->rpbx = c->tx - 2 * hx;
  c->rpby = c->cy * c->ty - 2 * hy;  // one y halo per cluster tile
  c->shape3p = ots::shape3p_index(c->E, c->bx, c->by);
  // the packed kernel's branch-free zero ring needs n0 % 4 == 0
  c->packed = p.stream_impl != 1 && c->cy == 1 && T <= ots::kMaxT3p && pl->K &&
              pl->geo.real_size % 4 == 0 && c->shape3p >= 0 &&
              pl->K->stream3p[T][c->shape3p] != nullptr;
  const int maxthr = c->packed ? 512 : (T * c->E >= 8 ? 256 : 512);
  if (c->bx != 8 && c->bx != 16 && c->bx != 32)
    return fail(OTS_ERR_UNSUPPORTED, "stream kernel block x must be 8, 16 or 32 (got %d)", c->bx);
  if ((c->bx * c->by) % 32 != 0)
    return fail(OTS_ERR_UNSUPPORTED,
                "stream kernel needs whole warps (block %d x %d is not a multiple of 32 threads)",
                c->bx, c->by);
  if (c->bx * c->by > maxthr)
    return fail(OTS_ERR_BLOCK_TOO_LARGE, "Block dimensions are too large! (%d x %d > %d threads)",
                c->bx, c->by, maxthr);
  if (c->tx > 256 || c->ty > 256)
    return fail(OTS_ERR_UNSUPPORTED, "stream tile %d x %d exceeds the 256-cell TMA box", c->tx,
                c->ty);
  if (c->rpbx < 4 || c->rpby < 1)
    return fail(OTS_ERR_INVALID_GEOMETRY,
                "Consistency error! stream tile %d x %d leaves no interior at T=%d", c->tx, c->ty,
                T);
  c->smem = c->packed ? ots::stream3p_smem_bytes(T, c->tx, c->ty, c->by, pl->info->na) + 128
                      : ots::stream_smem_bytes(T, c->tx, c->ty, c->cy, pl->info->na);
  if (c->smem > pl->smem_optin)
    return fail(OTS_ERR_SMEM_TOO_LARGE,
                "Not enough local memory for even one block! (%zu > %zu bytes)", c->smem,
                pl->smem_optin);
  const int n = pl->geo.real_size;
  c->nbx = ceil_div(n, c->rpbx);
  c->nby = ceil_div(n, c->rpby);
  int per_sm = 1;
  if (c->packed) {
    int b = 0;
    if (pl->K->stream3p_occ[T][c->shape3p](&b, c->bx * c->by, c->smem) == cudaSuccess && b > 0)
      per_sm = b;
  } else if (pl->K && pl->K->stream_occ[T][eidx]) {
    int b = 0;
    if (pl->K->stream_occ[T][eidx](&b, c->bx * c->by, c->smem, c->cy > 1) == cudaSuccess && b > 0)
      per_sm = b;
  }
  // Grid schedule: (tile, z segment) with tiles fastest.  The segment count
  // trades the T-plane pipeline fill of each segment against whole waves of
  // resident CTAs.
  const int64_t work = (int64_t)c->nbx * c->nby * n;
  const int slots = std::max(1, pl->sm_count) * per_sm;
  const int xy = c->nbx * c->nby * c->cy;  // CTAs per z segment
  double best = 1e300;
  int best_seg = n;
  for (int nseg = 1; nseg <= std::max(1, n / std::max(1, 2 * T)); ++nseg) {
    const int zseg = ceil_div(n, nseg);
    const int segs = ceil_div(n, zseg);
    const int waves = ceil_div(xy * segs, slots);
    const double cost = (double)waves * (zseg + 2 * T);
    if (cost < best * 0.999) {
      best = cost;
      best_seg = zseg;
    }
  }
  c->zseg = best_seg;
  c->nbz = ceil_div(n, c->zseg);
  c->work = work;
  c->chunk = 0;
  c->grid = xy * c->nbz;
  if ((int64_t)c->nbz * c->cy > 65535)
    return fail(OTS_ERR_INVALID_GEOMETRY, "stream grid too large along y (%d segments x %d)",
                c->nbz, c->cy);
  return OTS_OK;
}

// 3D tiled tensor map over one dense field; box = one stream tile plane.
ots_status make_tmap(const ots_plan* pl, const StreamCfg& c, const float* base, CUtensorMap* out) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return fail(OTS_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const ots::Layout& L = pl->L;
  cuuint64_t dims[3] = {(cuuint64_t)L.n0, (cuuint64_t)L.n1, (cuuint64_t)L.n2};
  cuuint64_t strides[2] = {(cuuint64_t)L.sy * 4, (cuuint64_t)L.sz * 4};
  cuuint32_t box[3] = {(cuuint32_t)c.tx, (cuuint32_t)c.ty, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = enc(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(OTS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OTS_OK;
}

// Resolve the kernel family and validate the tile launch.
ots_status resolve_kernel(ots_plan* pl, int requested, int* out) {
  const ots_params& p = pl->prm;
  const StencilInfo& si = *pl->info;
  const bool star_ok = si.star && si.dims == 3 &&
                       !(p.stencil == OTS_POISSON_3D && p.variant == OTS_VARIANT_REF);
  const bool star2d_ok = si.dims == 2 && (star2d_usable(pl) || (pl->K && pl->K->stream2dg[1]));
  int k = requested == OTS_KERNEL_AUTO ? p.kernel : requested;
  if (k == OTS_KERNEL_AUTO)
    k = (star_ok && p.block_z == 1 && p.engine == OTS_ENGINE_NATIVE) ? OTS_KERNEL_STREAM
                                                                      : OTS_KERNEL_TILE;
  const bool s1_ok = si.dims == 1 && pl->K && pl->K->stream1d[0];
  if (k == OTS_KERNEL_STREAM && !star_ok && !star2d_ok && !s1_ok)
    return fail(OTS_ERR_UNSUPPORTED,
                "stream kernel covers the 2D stencils and the 3D star stencils (jacobi-3d, "
                "poisson-3d in the baseline variant, gradient-3d)");
  if (k == OTS_KERNEL_TEX &&
      (si.dims != 2 || si.ns != 1 || p.elements_per_thread < 1 ||
       p.elements_per_thread > ots::kTexMaxE || !pl->K->tex[p.elements_per_thread]))
    return fail(OTS_ERR_UNSUPPORTED,
                "texture kernel covers 2D single-field stencils with E <= %d", ots::kTexMaxE);
  *out = k;
  return OTS_OK;
}

// Texture objects over field 0 of both state buffers (pitch-linear 2D, border
// addressing: a fetch outside the interior reads 0, the Dirichlet ring).
ots_status make_textures(ots_plan* pl) {
  if (pl->tex_ok) return OTS_OK;
  int align = 0, maxw = 0, maxh = 0;
  cudaDeviceGetAttribute(&align, cudaDevAttrTexturePitchAlignment, pl->device);
  cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxTexture2DLinearWidth, pl->device);
  cudaDeviceGetAttribute(&maxh, cudaDevAttrMaxTexture2DLinearHeight, pl->device);
  const size_t pitch = (size_t)pl->L.sy * sizeof(float);
  if (align <= 0 || pitch % (size_t)align != 0 || pl->L.n0 > maxw || pl->L.n1 > maxh)
    return fail(OTS_ERR_UNSUPPORTED, "texture kernel: %d x %d grid (pitch %zu) exceeds the "
                "2D linear texture limits (%d x %d, pitch alignment %d)",
                pl->L.n0, pl->L.n1, pitch, maxw, maxh, align);
  for (int b = 0; b < 2; ++b) {
    if (reinterpret_cast<uintptr_t>(pl->state[b][0]) % (uintptr_t)align != 0)
      return fail(OTS_ERR_UNSUPPORTED, "texture kernel: misaligned state buffer");
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = pl->state[b][0];
    rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
    rd.res.pitch2D.width = (size_t)pl->L.n0;
    rd.res.pitch2D.height = (size_t)pl->L.n1;
    rd.res.pitch2D.pitchInBytes = pitch;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeBorder;
    td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    OTS_CUDA(cudaCreateTextureObject(&pl->tex[b], &rd, &td, nullptr), "cudaCreateTextureObject");
  }
  pl->tex_ok = true;
  return OTS_OK;
}

ots_status validate_tile(ots_plan* pl) {
  const ots_params& p = pl->prm;
  ots_geometry& g = pl->geo;
  const int d = g.dims;
  for (int a = 0; a < d; ++a)
    if (g.real_per_block[a] < 1)
      return fail(OTS_ERR_INVALID_GEOMETRY,
                  "Consistency error! real per block along axis %d is %d (T=%d too deep for "
                  "the block)",
                  a, g.real_per_block[a], p.time_tile);
  const int threads = g.threads[0] * g.threads[1] * g.threads[2];
  if (threads > 1024)
    return fail(OTS_ERR_BLOCK_TOO_LARGE, "Block dimensions are too large! (%d threads)", threads);
  const int maxE = d == 3 ? ots::kMaxE3 : ots::kMaxE;
  if (p.elements_per_thread > maxE)
    return fail(OTS_ERR_UNSUPPORTED, "elements per thread %d > %d", p.elements_per_thread, maxE);
  if (!pl->K->tile[g.e_axis][p.elements_per_thread])
    return fail(OTS_ERR_UNSUPPORTED, "no tile instantiation for E=%d", p.elements_per_thread);
  cudaFuncAttributes fa{};
  if (pl->K->tile_attr[g.e_axis][p.elements_per_thread](&fa) == cudaSuccess &&
      threads > fa.maxThreadsPerBlock)
    return fail(OTS_ERR_BLOCK_TOO_LARGE,
                "Block dimensions are too large! (%d threads; the E=%d kernel takes at most %d)",
                threads, p.elements_per_thread, fa.maxThreadsPerBlock);
  const StencilInfo& si = *pl->info;
  const int Lx = g.comps[0] + 2 * si.rx, Ly = g.comps[1] + 2 * si.ry, Lz = g.comps[2] + 2 * si.rz;
  pl->tile_smem = (size_t)(2 * si.ns + (si.two_phase ? 1 : 0)) * Lx * Ly * Lz * sizeof(float);
  if (pl->tile_smem > pl->smem_optin)
    return fail(OTS_ERR_SMEM_TOO_LARGE, "Not enough local memory for even one block! (%zu > %zu)",
                pl->tile_smem, pl->smem_optin);
  for (int a = 0; a < 3; ++a)
    if (g.num_blocks[a] > (a == 0 ? 2147483647 : 65535))
      return fail(OTS_ERR_INVALID_GEOMETRY, "grid too large along axis %d", a);
  pl->tile_grid = dim3(g.num_blocks[0], g.num_blocks[1], g.num_blocks[2]);
  pl->tile_block = dim3(g.threads[0], g.threads[1], g.threads[2]);
  g.shared_bytes = (int64_t)pl->tile_smem;
  return OTS_OK;
}

void fill_geometry_for_kernel(ots_plan* pl) {
  ots_geometry& g = pl->geo;
  g.kernel = pl->prm.kernel;
  g.sm_count = pl->sm_count;
  cudaFuncAttributes a{};
  if (g.kernel == OTS_KERNEL_STREAM && g.dims == 1) {
    const Stream1dCfg& c = pl->s1cfg;
    g.comps[0] = 32 * c.V;
    g.comps[1] = g.comps[2] = 1;
    g.real_per_block[0] = c.rpb;
    g.real_per_block[1] = g.real_per_block[2] = 1;
    g.num_blocks[0] = c.nw;
    g.num_blocks[1] = g.num_blocks[2] = 1;
    g.threads[0] = 32;  // one warp per strip
    g.threads[1] = g.threads[2] = 1;
    g.e_axis = 0;
    g.shared_bytes = 0;
    g.useful_ratio = (double)pl->geo.real_size / ((double)32 * c.V * c.nw);
    if (pl->K->stream1d_attr[c.vidx] && pl->K->stream1d_attr[c.vidx](&a) == cudaSuccess)
      g.registers = a.numRegs;
    if (g.registers > 0)
      g.ctas_per_sm = std::min(32, 65536 / (ots::kStream1dThreads * ((g.registers + 7) / 8 * 8)));
  } else if (g.kernel == OTS_KERNEL_STREAM && g.dims == 2) {
    const Stream2dCfg& c = pl->s2cfg;
    g.comps[0] = ots::kStream2dWidth;
    g.comps[1] = c.zseg + 2 * c.R * c.T;
    g.comps[2] = 1;
    g.real_per_block[0] = c.rpbx;
    g.real_per_block[1] = c.zseg;
    g.real_per_block[2] = 1;
    g.num_blocks[0] = c.ntx;
    g.num_blocks[1] = c.nseg;
    g.num_blocks[2] = 1;
    g.threads[0] = 32;  // one warp per strip segment
    g.threads[1] = 1;
    g.threads[2] = 1;
    g.e_axis = 0;
    g.shared_bytes = 0;
    {
      const double n = pl->geo.real_size;
      g.useful_ratio = (n * n) / ((double)ots::kStream2dWidth * c.ntx * c.nseg *
                                  (double)(c.zseg + 2 * c.R * c.T));
    }
    if (c.generic) {
      auto attr = pl->K->stream2dg_attr[c.T];
      if (attr && attr(&a, pl->prm.variant == OTS_VARIANT_FAST) == cudaSuccess)
        g.registers = a.numRegs;
    } else {
      auto attr = c.packed ? pl->K->stream2dp_attr[c.T] : pl->K->stream2d_attr[c.T];
      if (attr && attr(&a) == cudaSuccess) g.registers = a.numRegs;
    }
    g.ctas_per_sm = c.warps_per_sm / (ots::kStream2dThreads / 32);
  } else if (g.kernel == OTS_KERNEL_STREAM) {
    const StreamCfg& c = pl->scfg;
    g.comps[0] = c.tx;
    g.comps[1] = c.cy * c.ty;  // a cluster's CTAs share one tile
    g.comps[2] = c.zseg + 2 * c.T;
    g.real_per_block[0] = c.rpbx;
    g.real_per_block[1] = c.rpby;
    g.real_per_block[2] = c.zseg;
    g.num_blocks[0] = c.nbx;
    g.num_blocks[1] = c.nby;
    g.num_blocks[2] = c.nbz;
    g.threads[0] = c.bx;
    g.threads[1] = c.by;
    g.threads[2] = 1;
    g.e_axis = 1;
    g.shared_bytes = (int64_t)c.smem;
    {
      const double n = pl->geo.real_size;
      g.useful_ratio = (n * n * n) / ((double)c.tx * c.cy * c.ty * c.nbx * c.nby *
                                      (double)c.nbz * (c.zseg + 2 * c.T));
    }
    int b = 0;
    if (c.packed) {
      if (pl->K->stream3p_attr[c.T][c.shape3p](&a) == cudaSuccess) g.registers = a.numRegs;
      if (pl->K->stream3p_occ[c.T][c.shape3p](&b, c.bx * c.by, c.smem) == cudaSuccess)
        g.ctas_per_sm = b;
    } else {
      if (pl->K->stream_attr[c.T][c.eidx] &&
          pl->K->stream_attr[c.T][c.eidx](&a, c.cy > 1) == cudaSuccess)
        g.registers = a.numRegs;
      if (pl->K->stream_occ[c.T][c.eidx] &&
          pl->K->stream_occ[c.T][c.eidx](&b, c.bx * c.by, c.smem, c.cy > 1) == cudaSuccess)
        g.ctas_per_sm = b;
    }
  } else if (g.kernel == OTS_KERNEL_PLAIN) {
    // one cell per thread, blocks of 256 x 1 (1D) or 32 x 8 x 1, one step
    // per launch, no shared memory and no redundant cells
    const int bx = g.dims == 1 ? 256 : 32, by = g.dims == 1 ? 1 : 8;
    const int n = pl->geo.real_size;
    g.threads[0] = bx;
    g.threads[1] = by;
    g.threads[2] = 1;
    g.comps[0] = g.real_per_block[0] = bx;
    g.comps[1] = g.real_per_block[1] = by;
    g.comps[2] = g.real_per_block[2] = 1;
    g.num_blocks[0] = ceil_div(n, bx);
    g.num_blocks[1] = g.dims >= 2 ? ceil_div(n, by) : 1;
    g.num_blocks[2] = g.dims == 3 ? n : 1;
    g.e_axis = 0;
    g.shared_bytes = 0;
    g.useful_ratio = 1.0;
    g.launches = pl->prm.time_steps;
    if (pl->K->plain_attr(&a) == cudaSuccess) g.registers = a.numRegs;
    if (a.numRegs > 0)
      g.ctas_per_sm = std::max(
          1, std::min(2048 / (bx * by), 65536 / (bx * by * ((a.numRegs + 7) / 8 * 8))));
  } else {
    const int E = pl->prm.elements_per_thread;
    if (g.kernel == OTS_KERNEL_TEX) {
      if (E <= ots::kTexMaxE && pl->K->tex_attr[E] && pl->K->tex_attr[E](&a) == cudaSuccess)
        g.registers = a.numRegs;
    } else if (pl->K->tile_attr[g.e_axis][E](&a) == cudaSuccess) {
      g.registers = a.numRegs;
    }
    // resident CTAs per SM from registers, shared memory and threads
    const int thr = g.threads[0] * g.threads[1] * g.threads[2];
    if (a.numRegs > 0 && thr > 0) {
      const int warps = (thr + 31) / 32;
      const int by_regs = 65536 / (warps * 32 * ((a.numRegs + 7) / 8 * 8));
      const int by_smem = pl->tile_smem ? (int)(233472 / (pl->tile_smem + 1024)) : 32;
      const int by_thr = 2048 / thr;
      g.ctas_per_sm = std::max(0, std::min(std::min(by_regs, by_smem), std::min(by_thr, 32)));
    }
  }
}

// --------------------------------------------------------------- launch --

ots::StepParams step_params(const ots_plan* pl, int in_buf, int base, int T) {
  ots::StepParams sp{};
  for (int f = 0; f < pl->info->ns; ++f) {
    sp.in[f] = pl->state[in_buf][f];
    sp.out[f] = pl->state[in_buf ^ 1][f];
  }
  for (int a = 0; a < pl->info->na; ++a) sp.aux[a] = pl->aux[a];
  sp.L = pl->L;
  sp.T = T;
  sp.steps = pl->prm.time_steps;
  sp.base_step = base;
  sp.phase_limit = pl->prm.phase_limit;
  sp.op = pl->op;
  for (int a = 0; a < 3; ++a) sp.rpb[a] = pl->geo.real_per_block[a];
  return sp;
}

ots_status enqueue_run(ots_plan* pl, int kernel) {
  const int S = pl->prm.time_steps;
  if (S == 0) return OTS_OK;
  cudaError_t e = cudaSuccess;
  if (kernel == OTS_KERNEL_PLAIN) {
    dim3 b(pl->geo.dims == 1 ? 256 : 32, pl->geo.dims == 1 ? 1 : 8, 1);
    dim3 g(ceil_div(pl->L.n0, b.x), ceil_div(pl->L.n1, b.y), pl->L.n2);
    for (int s = 0; s < S && e == cudaSuccess; ++s) {
      ots::StepParams sp = step_params(pl, pl->cur, s, 1);
      e = pl->K->plain(sp, g, b, 0, pl->stream);
      pl->cur ^= 1;
    }
  } else if (kernel == OTS_KERNEL_STREAM && pl->geo.dims == 1) {
    const int T = pl->prm.time_tile;
    const Stream1dCfg& c = pl->s1cfg;
    for (int base = 0; base < S && e == cudaSuccess; base += T) {
      ots::Stream1dParams sp{};
      sp.in = pl->state[pl->cur][0];
      sp.out = pl->state[pl->cur ^ 1][0];
      sp.n = pl->L.n0;
      sp.T = std::min(T, S - base);  // the halo of T covers a shallower last launch
      sp.base_step = base;
      sp.rpb = c.rpb;
      sp.hx = c.hx;
      sp.nw = c.nw;
      sp.op = pl->op;
      e = pl->K->stream1d[c.vidx](sp, dim3(c.grid), pl->stream);
      pl->cur ^= 1;
    }
  } else if (kernel == OTS_KERNEL_STREAM && pl->geo.dims == 2) {
    const int T = pl->prm.time_tile;
    for (int base = 0; base < S && e == cudaSuccess; base += T) {
      const int Tl = std::min(T, S - base);
      Stream2dCfg c = pl->s2cfg;
      if (Tl != c.T) {
        ots_status st = derive_stream2d(pl, Tl, &c);
        if (st != OTS_OK) return st;
      }
      if (c.generic) {
        ots::Stream2dgParams sp{};
        for (int f = 0; f < pl->info->ns; ++f) {
          sp.in[f] = pl->state[pl->cur][f];
          sp.out[f] = pl->state[pl->cur ^ 1][f];
        }
        for (int a = 0; a < pl->info->na; ++a) sp.aux[a] = pl->aux[a];
        sp.L = pl->L;
        sp.ntx = c.ntx;
        sp.nseg = c.nseg;
        sp.zseg = c.zseg;
        sp.base_step = base;
        sp.op = pl->op;
        e = pl->K->stream2dg[Tl](sp, dim3(c.grid), pl->stream);
      } else {
        ots::Stream2dParams sp{};
        sp.in = pl->state[pl->cur][0];
        sp.out = pl->state[pl->cur ^ 1][0];
        sp.aux = pl->info->na ? pl->aux[0] : nullptr;
        sp.L = pl->L;
        sp.ntx = c.ntx;
        sp.nseg = c.nseg;
        sp.zseg = c.zseg;
        sp.base_step = base;
        sp.op = pl->op;
        e = (c.packed ? pl->K->stream2dp[Tl] : pl->K->stream2d[Tl])(sp, dim3(c.grid),
                                                                     pl->stream);
      }
      pl->cur ^= 1;
    }
  } else if (kernel == OTS_KERNEL_STREAM) {
    const int T = pl->prm.time_tile;
    for (int base = 0; base < S && e == cudaSuccess; base += T) {
      const int Tl = std::min(T, S - base);
      StreamCfg c = pl->scfg;
      if (Tl != c.T) {
        ots_status st = derive_stream(pl, Tl, &c);
        if (st != OTS_OK) return st;
      }
      ots::StreamParams sp{};
      sp.out = pl->state[pl->cur ^ 1][0];
      sp.aux = pl->info->na ? pl->aux[0] : nullptr;
      sp.L = pl->L;
      sp.ntx = c.nbx;
      sp.nty = c.nby;
      sp.work = c.work;
      sp.chunk = c.chunk;
      sp.zseg = c.zseg;
      sp.cy = c.cy;
      sp.base_step = base;
      sp.err = pl->d_err;
      sp.wait_ns = pl->wait_ns;
      sp.hold_plane = pl->hold_plane;
      sp.op = pl->op;
      CUtensorMap m;
      if (Tl == pl->scfg.T) {
        m = pl->tmap[pl->cur];
        if (pl->info->na) sp.amap = pl->amap;
      } else {
        // the last, shallower launch has its own tile box
        ots_status st = make_tmap(pl, c, pl->state[pl->cur][0], &m);
        if (st == OTS_OK && pl->info->na) st = make_tmap(pl, c, pl->aux[0], &sp.amap);
        if (st != OTS_OK) return st;
      }
      if (c.packed)
        e = pl->K->stream3p[Tl][c.shape3p](m, sp, dim3(c.nbx * c.nby, c.nbz, 1),
                                           dim3(c.bx, c.by, 1), c.smem, pl->stream);
      else
        e = pl->K->stream[Tl][c.eidx](m, sp, dim3(c.nbx * c.nby, c.nbz * c.cy, 1),
                                      dim3(c.bx, c.by, 1), c.smem, pl->stream);
      pl->cur ^= 1;
    }
  } else if (kernel == OTS_KERNEL_TEX) {
    const int T = pl->prm.time_tile;
    auto fn = pl->K->tex[pl->prm.elements_per_thread];
    for (int base = 0; base < S && e == cudaSuccess; base += T) {
      ots::StepParams sp = step_params(pl, pl->cur, base, T);
      sp.tex = pl->tex[pl->cur];
      e = fn(sp, pl->tile_grid, pl->tile_block, pl->tile_smem, pl->stream);
      pl->cur ^= 1;
    }
  } else {
    const int T = pl->prm.time_tile;
    auto fn = pl->K->tile[pl->geo.e_axis][pl->prm.elements_per_thread];
    for (int base = 0; base < S && e == cudaSuccess; base += T) {
      ots::StepParams sp = step_params(pl, pl->cur, base, T);
      sp.clocks = pl->d_clocks;  // each launch overwrites: the last one stays
      e = fn(sp, pl->tile_grid, pl->tile_block, pl->tile_smem, pl->stream);
      pl->cur ^= 1;
    }
  }
  pl->clocks_valid = pl->d_clocks && kernel == OTS_KERNEL_TILE;
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  return OTS_OK;
}

ots_status check_err_word(ots_plan* pl) {
  int h = 0;
  OTS_CUDA(cudaMemcpyAsync(&h, pl->d_err, sizeof(int), cudaMemcpyDeviceToHost, pl->stream),
           "read error word");
  OTS_CUDA(cudaStreamSynchronize(pl->stream), "synchronize");
  if (h != 0) {
    cudaMemsetAsync(pl->d_err, 0, sizeof(int), pl->stream);
    cudaStreamSynchronize(pl->stream);
    return fail(OTS_ERR_TIMEOUT, "a bounded device wait gave up (error word 0x%x)", h);
  }
  return OTS_OK;
}

// Host (reference layout, ring `pad`, pitch P) <-> device (dense, pitched).
ots_status copy_field(ots_plan* pl, float* dev, const float* host, bool to_dev, int pad, int P,
                      bool interior_only_host) {
  const ots::Layout& L = pl->L;
  const int d = pl->geo.dims;
  const size_t hp = interior_only_host ? (size_t)L.n0 : (size_t)P;   // host row pitch (floats)
  const size_t hplane = interior_only_host ? (size_t)L.n0 * L.n1 : (size_t)P * P;
  const size_t off = interior_only_host
                         ? 0
                         : (size_t)pad + (d >= 2 ? (size_t)pad * P : 0) +
                               (d == 3 ? (size_t)pad * P * P : 0);
  const cudaMemcpyKind kind = to_dev ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  // dense host array and unpadded device rows: one linear copy
  if (interior_only_host && L.sy == L.n0) {
    const size_t bytes = (size_t)L.n0 * L.n1 * L.n2 * sizeof(float);
    if (to_dev)
      OTS_CUDA(cudaMemcpyAsync(dev, host, bytes, kind, pl->stream), "upload");
    else
      OTS_CUDA(cudaMemcpyAsync((float*)host, dev, bytes, kind, pl->stream), "download");
    return OTS_OK;
  }
  if (d == 1) {
    if (to_dev)
      OTS_CUDA(cudaMemcpyAsync(dev, host + off, L.n0 * sizeof(float), kind, pl->stream), "upload");
    else
      OTS_CUDA(cudaMemcpyAsync((float*)host + off, dev, L.n0 * sizeof(float), kind, pl->stream),
               "download");
    return OTS_OK;
  }
  if (d == 2) {
    if (to_dev)
      OTS_CUDA(cudaMemcpy2DAsync(dev, L.sy * sizeof(float), host + off, hp * sizeof(float),
                                 L.n0 * sizeof(float), L.n1, kind, pl->stream),
               "upload");
    else
      OTS_CUDA(cudaMemcpy2DAsync((float*)host + off, hp * sizeof(float), dev, L.sy * sizeof(float),
                                 L.n0 * sizeof(float), L.n1, kind, pl->stream),
               "download");
    return OTS_OK;
  }
  cudaMemcpy3DParms m{};
  cudaPitchedPtr hptr =
      make_cudaPitchedPtr((void*)(host + off), hp * sizeof(float), L.n0, hplane / hp);
  cudaPitchedPtr dptr = make_cudaPitchedPtr(dev, L.sy * sizeof(float), L.n0, L.sz / L.sy);
  m.extent = make_cudaExtent(L.n0 * sizeof(float), L.n1, L.n2);
  m.kind = kind;
  if (to_dev) {
    m.srcPtr = hptr;
    m.dstPtr = dptr;
  } else {
    m.srcPtr = dptr;
    m.dstPtr = hptr;
  }
  OTS_CUDA(cudaMemcpy3DAsync(&m, pl->stream), to_dev ? "upload" : "download");
  return OTS_OK;
}

void free_plan(ots_plan* pl) {
  if (!pl) return;
  cudaSetDevice(pl->device);
  for (int b = 0; b < 2; ++b)
    for (int f = 0; f < 3; ++f)
      if (pl->state[b][f]) cudaFree(pl->state[b][f]);
  for (int a = 0; a < 2; ++a)
    if (pl->aux[a]) cudaFree(pl->aux[a]);
  if (pl->d_err) cudaFree(pl->d_err);
  if (pl->d_clocks) cudaFree(pl->d_clocks);
  for (int b = 0; b < 2; ++b)
    if (pl->tex[b]) cudaDestroyTextureObject(pl->tex[b]);
  if (pl->ev0) cudaEventDestroy(pl->ev0);
  if (pl->ev1) cudaEventDestroy(pl->ev1);
  if (pl->stream) cudaStreamDestroy(pl->stream);
  delete pl;
}

}  // namespace

// ====================================================================== ABI

extern "C" {

const char* ots_last_error(void) { return g_last_error.c_str(); }

const char* ots_status_string(ots_status s) {
  switch (s) {
    case OTS_OK: return "OK";
    case OTS_ERR_INVALID_ARGUMENT: return "invalid argument";
    case OTS_ERR_INVALID_GEOMETRY: return "invalid geometry";
    case OTS_ERR_SMEM_TOO_LARGE: return "shared memory too large";
    case OTS_ERR_BLOCK_TOO_LARGE: return "block too large";
    case OTS_ERR_CUDA: return "CUDA error";
    case OTS_ERR_TIMEOUT: return "device wait timed out";
    case OTS_ERR_UNSUPPORTED: return "unsupported";
    case OTS_ERR_NO_DEVICE: return "no CUDA device";
    case OTS_ERR_OUT_OF_MEMORY: return "out of device memory";
  }
  return "unknown status";
}

ots_status ots_device_info(int32_t device, char* name, size_t name_len, int32_t* sm_count,
                           int64_t* smem_per_block, int64_t* global_mem) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(OTS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= n) return fail(OTS_ERR_INVALID_ARGUMENT, "device %d out of range", device);
  cudaDeviceProp prop;
  OTS_CUDA(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (name && name_len) snprintf(name, name_len, "%s", prop.name);
  if (sm_count) *sm_count = prop.multiProcessorCount;
  if (smem_per_block) *smem_per_block = (int64_t)prop.sharedMemPerBlockOptin;
  if (global_mem) *global_mem = (int64_t)prop.totalGlobalMem;
  return OTS_OK;
}

const char* ots_stencil_name(int32_t s) {
  return (s >= 0 && s < OTS_NUM_STENCILS) ? kInfo[s].name : nullptr;
}

int32_t ots_stencil_from_name(const char* name) {
  if (!name) return -1;
  for (int s = 0; s < OTS_NUM_STENCILS; ++s)
    if (strcmp(name, kInfo[s].name) == 0) return s;
  return -1;
}

int32_t ots_stencil_dims(int32_t s) { return (s >= 0 && s < OTS_NUM_STENCILS) ? kInfo[s].dims : 0; }
int32_t ots_stencil_num_fields(int32_t s) {
  return (s >= 0 && s < OTS_NUM_STENCILS) ? kInfo[s].ns : 0;
}
int32_t ots_stencil_num_aux(int32_t s) {
  return (s >= 0 && s < OTS_NUM_STENCILS) ? kInfo[s].na : 0;
}

ots_status ots_stencil_model_constants(int32_t s, double out[8]) {
  if (s < 0 || s >= OTS_NUM_STENCILS) return fail(OTS_ERR_INVALID_ARGUMENT, "unknown stencil id %d", s);
  if (!out) return fail(OTS_ERR_INVALID_ARGUMENT, "out is NULL");
  if (kInfo[s].r5[0] < 0)
    return fail(OTS_ERR_UNSUPPORTED, "the %s runner prints no model constants", kInfo[s].name);
  for (int i = 0; i < 8; ++i) out[i] = kInfo[s].r5[i];
  return OTS_OK;
}

ots_status ots_fill_reference(int32_t dims, int32_t P, int32_t padding, int32_t real_size,
                              uint32_t seed, float* const* fields, int32_t nf) {
  if (dims < 1 || dims > 3 || P < 1 || !fields || nf < 1)
    return fail(OTS_ERR_INVALID_ARGUMENT, "bad fill arguments");
  for (int f = 0; f < nf; ++f)
    if (!fields[f]) return fail(OTS_ERR_INVALID_ARGUMENT, "fill field %d is NULL", f);
  srand(seed);
  const int PZ = dims == 3 ? P : 1, PY = dims >= 2 ? P : 1;
  const int lo = padding, hi = padding + real_size;
  for (int z = 0; z < PZ; ++z)
    for (int y = 0; y < PY; ++y)
      for (int x = 0; x < P; ++x) {
        const size_t i = ((size_t)z * PY + y) * P + x;
        const bool in = x >= lo && x < hi && (dims < 2 || (y >= lo && y < hi)) &&
                        (dims < 3 || (z >= lo && z < hi));
        for (int f = 0; f < nf; ++f)
          fields[f][i] = in ? (float)rand() / ((float)RAND_MAX + 1.0f) : 0.0f;
      }
  return OTS_OK;
}

// The synthetic image of the Rician / TV workloads.  Uniform deviates come
// from a SplitMix64 stream (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014) as 53-bit doubles, normal
// deviates from the Box-Muller transform of two uniforms.
namespace {
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
};
}  // namespace

ots_status ots_fill_disks(int32_t n, uint64_t seed, int32_t count, float background, float sigma,
                          float* noisy, float* clean) {
  if (n < 1 || count < 0 || !noisy || !(sigma >= 0.0f))
    return fail(OTS_ERR_INVALID_ARGUMENT, "bad disk-image arguments");
  SplitMix64 rng{seed};
  std::vector<double> img((size_t)n * n, (double)background);
  for (int d = 0; d < count; ++d) {
    const double cx = rng.uniform() * n, cy = rng.uniform() * n;
    const double r = n / 64.0 + rng.uniform() * (n / 12.0 - n / 64.0);
    const double val = 0.2 + rng.uniform() * 0.8;
    const int y0 = std::max(0, (int)(cy - r) - 1), y1 = std::min(n, (int)(cy + r) + 2);
    const int x0 = std::max(0, (int)(cx - r) - 1), x1 = std::min(n, (int)(cx + r) + 2);
    for (int y = y0; y < y1; ++y)
      for (int x = x0; x < x1; ++x)
        if ((x - cx) * (x - cx) + (y - cy) * (y - cy) <= r * r) img[(size_t)y * n + x] = val;
  }
  const double two_pi = 6.283185307179586;
  for (size_t i = 0; i < img.size(); ++i) {
    const double u1 = 1.0 - rng.uniform(), u2 = rng.uniform();  // u1 in (0, 1]
    const double rad = std::sqrt(-2.0 * std::log(u1));
    const double n1 = sigma * rad * std::cos(two_pi * u2), n2 = sigma * rad * std::sin(two_pi * u2);
    const double a = img[i] + n1;
    noisy[i] = (float)std::sqrt(a * a + n2 * n2);
    if (clean) clean[i] = (float)img[i];
  }
  return OTS_OK;
}

static ots_status prepare(const ots_params* params, ots_plan* pl);

ots_status ots_derive_geometry(const ots_params* params, ots_geometry* out) {
  if (!out) return fail(OTS_ERR_INVALID_ARGUMENT, "geometry output is NULL");
  const StencilInfo* si = nullptr;
  ots_status st = derive(params, out, &si);
  if (st != OTS_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return OTS_OK;  // no device: the reference derivation only
  }
  // with a device: resolve and validate the kernel as ots_plan_create would
  ots_plan tmp;
  st = prepare(params, &tmp);
  if (st != OTS_OK) return st;
  *out = tmp.geo;
  return OTS_OK;
}

// Everything plan creation does short of allocating: geometry, operator
// arguments, kernel resolution and launch validation, device layout.
static ots_status prepare(const ots_params* params, ots_plan* pl) {
  ots_status st = derive(params, &pl->geo, &pl->info);
  if (st != OTS_OK) return st;
  pl->prm = *params;
  pl->K = &ots::kernels_for(params->stencil);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(OTS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (params->device < 0 || params->device >= ndev)
    return fail(OTS_ERR_INVALID_ARGUMENT, "device %d out of range", params->device);
  pl->device = params->device;
  cudaError_t ce = cudaSetDevice(pl->device);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaSetDevice");
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, pl->device);
  pl->sm_count = prop.multiProcessorCount;
  pl->smem_optin = prop.sharedMemPerBlockOptin;

  // op arguments
  const ots_params& p = pl->prm;
  pl->op.variant = p.variant;
  float coef = p.coef;
  if (coef == 0.0f) {
    switch (p.stencil) {
      case OTS_JACOBI_1D: coef = 0.333f; break;                   // jacobi-1d.cpp:635
      case OTS_JACOBI_1D_5PT: coef = 0.2f; break;                 // jacobi-1d-5pt.cpp:509
      case OTS_JACOBI_1D_7PT: coef = 0.2f; break;                 // jacobi-1d-7pt.cpp:517
      case OTS_JACOBI_2D: coef = 1.0f / 5.0f; break;              // jacobi-2d.cpp:825
      case OTS_JACOBI_3D:                                         // jacobi-3d.cpp:304
        coef = p.variant == OTS_VARIANT_REF ? 0.143f : (float)(1.0 / 7.0);
        break;
      default: break;
    }
  }
  pl->op.coef = coef;
  float h2 = p.h2;
  if (h2 == 0.0f && pl->geo.real_size > 1) {
    const double h = 1.0 / (double)(pl->geo.real_size - 1);
    h2 = (float)(h * h);
  }
  pl->op.h2 = h2;
  pl->geo.coef = coef;
  pl->geo.h2 = h2;

  // kernel family + launch validation
  int k = 0;
  st = resolve_kernel(pl, OTS_KERNEL_AUTO, &k);
  if (st != OTS_OK) return st;
  pl->prm.kernel = k;
  if (k == OTS_KERNEL_STREAM && pl->geo.dims == 1) {
    st = derive_stream1d(pl, &pl->s1cfg);
  } else if (k == OTS_KERNEL_STREAM && pl->geo.dims == 2) {
    st = derive_stream2d(pl, p.time_tile, &pl->s2cfg);
  } else if (k == OTS_KERNEL_STREAM) {
    st = derive_stream(pl, p.time_tile, &pl->scfg);
  } else if (k == OTS_KERNEL_TILE || k == OTS_KERNEL_TEX) {
    st = validate_tile(pl);
  }
  if (st != OTS_OK) return st;

  // device layout: interior only, rows padded to 32 floats
  const int d = pl->geo.dims, n = pl->geo.real_size;
  pl->L.n0 = n;
  pl->L.n1 = d >= 2 ? n : 1;
  pl->L.n2 = d == 3 ? n : 1;
  pl->L.sy = round_up(n, 32);
  pl->L.sz = pl->L.sy * pl->L.n1;
  pl->field_elems = pl->L.sz * pl->L.n2;
  fill_geometry_for_kernel(pl);
  return OTS_OK;
}

ots_status ots_plan_create(const ots_params* params, ots_plan** out) {
  if (!out) return fail(OTS_ERR_INVALID_ARGUMENT, "plan output is NULL");
  if (!params) return fail(OTS_ERR_INVALID_ARGUMENT, "params is NULL");
  *out = nullptr;
  ots_plan* pl = new ots_plan();
  ots_status st = prepare(params, pl);
  if (st != OTS_OK) {
    delete pl;
    return st;
  }
  const int k = pl->prm.kernel;
  cudaError_t ce;
  ce = cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaEventCreate(&pl->ev0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&pl->ev1);
  if (ce == cudaSuccess) ce = cudaMalloc(&pl->d_err, sizeof(int));
  if (ce == cudaSuccess) ce = cudaMemset(pl->d_err, 0, sizeof(int));
  const size_t bytes = (size_t)pl->field_elems * sizeof(float);
  for (int b = 0; b < 2 && ce == cudaSuccess; ++b)
    for (int f = 0; f < pl->info->ns && ce == cudaSuccess; ++f) {
      ce = cudaMalloc(&pl->state[b][f], bytes);
      if (ce == cudaSuccess) ce = cudaMemset(pl->state[b][f], 0, bytes);
    }
  for (int a = 0; a < pl->info->na && ce == cudaSuccess; ++a) {
    ce = cudaMalloc(&pl->aux[a], bytes);
    if (ce == cudaSuccess) ce = cudaMemset(pl->aux[a], 0, bytes);
  }
  if (ce != cudaSuccess) {
    ots_status s2 = cuda_fail(ce, "plan allocation");
    free_plan(pl);
    return s2;
  }
  if (k == OTS_KERNEL_STREAM && pl->geo.dims == 3) {
    st = make_tmap(pl, pl->scfg, pl->state[0][0], &pl->tmap[0]);
    if (st == OTS_OK) st = make_tmap(pl, pl->scfg, pl->state[1][0], &pl->tmap[1]);
    if (st == OTS_OK && pl->info->na) st = make_tmap(pl, pl->scfg, pl->aux[0], &pl->amap);
    if (st != OTS_OK) {
      free_plan(pl);
      return st;
    }
    pl->tmap_ok = true;
  }
  if (k == OTS_KERNEL_TEX) {
    st = make_textures(pl);
    if (st != OTS_OK) {
      free_plan(pl);
      return st;
    }
  }
  *out = pl;
  return OTS_OK;
}

void ots_plan_destroy(ots_plan* plan) { free_plan(plan); }

ots_status ots_plan_geometry(const ots_plan* plan, ots_geometry* out) {
  if (!plan || !out) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  *out = plan->geo;
  return OTS_OK;
}

static ots_status upload_impl(ots_plan* pl, const float* const* state, const float* const* aux,
                              bool interior, bool wait = true) {
  if (!pl || !state) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  OTS_CUDA(cudaSetDevice(pl->device), "cudaSetDevice");
  for (int f = 0; f < pl->info->ns; ++f) {
    if (!state[f]) return fail(OTS_ERR_INVALID_ARGUMENT, "state field %d is NULL", f);
    ots_status s = copy_field(pl, pl->state[0][f], state[f], true, pl->geo.padding,
                              pl->geo.padded_size, interior);
    if (s != OTS_OK) return s;
    // Every launch writes every interior cell of its output buffer, so the
    // second ping-pong buffer's contents are never read before they are
    // overwritten.  Only phase-limited kernels (-p 1/2/3) stop before their
    // write-back; for them the second buffer gets the input too, as the
    // reference writes its input to both buffers
    // (opencl/jacobi-2d/jacobi-2d.cpp:874-886).
    if (pl->prm.phase_limit != 0)
      OTS_CUDA(cudaMemcpyAsync(pl->state[1][f], pl->state[0][f],
                               (size_t)pl->field_elems * sizeof(float),
                               cudaMemcpyDeviceToDevice, pl->stream),
               "device copy");
  }
  for (int a = 0; a < pl->info->na; ++a) {
    if (!aux || !aux[a]) return fail(OTS_ERR_INVALID_ARGUMENT, "aux field %d is NULL", a);
    ots_status s = copy_field(pl, pl->aux[a], aux[a], true, pl->geo.padding, pl->geo.padded_size,
                              interior);
    if (s != OTS_OK) return s;
  }
  pl->cur = 0;
  if (wait) OTS_CUDA(cudaStreamSynchronize(pl->stream), "upload");
  return OTS_OK;
}

ots_status ots_upload(ots_plan* plan, const float* const* state, const float* const* aux) {
  return upload_impl(plan, state, aux, false);
}

ots_status ots_upload_interior(ots_plan* plan, const float* const* state, const float* const* aux) {
  return upload_impl(plan, state, aux, true);
}

ots_status ots_upload_async(ots_plan* plan, const float* const* state, const float* const* aux) {
  return upload_impl(plan, state, aux, false, false);
}

ots_status ots_upload_interior_async(ots_plan* plan, const float* const* state,
                                     const float* const* aux) {
  return upload_impl(plan, state, aux, true, false);
}

ots_status ots_run_async(ots_plan* plan, int32_t kernel) {
  if (!plan) return fail(OTS_ERR_INVALID_ARGUMENT, "plan is NULL");
  OTS_CUDA(cudaSetDevice(plan->device), "cudaSetDevice");
  int k = 0;
  ots_status st = resolve_kernel(plan, kernel, &k);
  if (st != OTS_OK) return st;
  if (k != plan->prm.kernel) {
    // a different family than the plan was built for: validate it now
    if (k == OTS_KERNEL_TILE) {
      st = validate_tile(plan);
    } else if (k == OTS_KERNEL_TEX) {
      st = validate_tile(plan);
      if (st == OTS_OK) st = make_textures(plan);
    } else if (k == OTS_KERNEL_STREAM && plan->geo.dims == 1) {
      if (plan->s1cfg.V == 0) st = derive_stream1d(plan, &plan->s1cfg);
    } else if (k == OTS_KERNEL_STREAM && plan->geo.dims == 2) {
      if (plan->s2cfg.T == 0) st = derive_stream2d(plan, plan->prm.time_tile, &plan->s2cfg);
    } else if (k == OTS_KERNEL_STREAM) {
      if (!plan->tmap_ok) {
        st = derive_stream(plan, plan->prm.time_tile, &plan->scfg);
        if (st == OTS_OK) st = make_tmap(plan, plan->scfg, plan->state[0][0], &plan->tmap[0]);
        if (st == OTS_OK) st = make_tmap(plan, plan->scfg, plan->state[1][0], &plan->tmap[1]);
        if (st == OTS_OK && plan->info->na)
          st = make_tmap(plan, plan->scfg, plan->aux[0], &plan->amap);
        if (st == OTS_OK) plan->tmap_ok = true;
      }
    }
    if (st != OTS_OK) return st;
  }
  return enqueue_run(plan, k);
}

ots_status ots_sync(ots_plan* plan) {
  if (!plan) return fail(OTS_ERR_INVALID_ARGUMENT, "plan is NULL");
  OTS_CUDA(cudaSetDevice(plan->device), "cudaSetDevice");
  OTS_CUDA(cudaStreamSynchronize(plan->stream), "synchronize");
  return check_err_word(plan);
}

ots_status ots_run(ots_plan* plan, int32_t kernel, ots_timing* timing) {
  if (!plan) return fail(OTS_ERR_INVALID_ARGUMENT, "plan is NULL");
  OTS_CUDA(cudaSetDevice(plan->device), "cudaSetDevice");
  OTS_CUDA(cudaStreamSynchronize(plan->stream), "synchronize");
  const auto t0 = std::chrono::steady_clock::now();
  OTS_CUDA(cudaEventRecord(plan->ev0, plan->stream), "event record");
  ots_status st = ots_run_async(plan, kernel);
  if (st != OTS_OK) return st;
  OTS_CUDA(cudaEventRecord(plan->ev1, plan->stream), "event record");
  OTS_CUDA(cudaEventSynchronize(plan->ev1), "kernel execution");
  const auto t1 = std::chrono::steady_clock::now();
  st = check_err_word(plan);
  if (st != OTS_OK) return st;
  if (timing) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, plan->ev0, plan->ev1);
    timing->event_ms = ms;
    timing->wall_s = std::chrono::duration<double>(t1 - t0).count();
    int k = 0;
    resolve_kernel(plan, kernel, &k);
    timing->launches = k == OTS_KERNEL_PLAIN ? plan->prm.time_steps : plan->geo.launches;
    timing->steps = plan->prm.time_steps;
  }
  return OTS_OK;
}

static ots_status download_impl(ots_plan* pl, float* const* state, bool interior,
                                bool wait = true) {
  if (!pl || !state) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  OTS_CUDA(cudaSetDevice(pl->device), "cudaSetDevice");
  for (int f = 0; f < pl->info->ns; ++f) {
    if (!state[f]) return fail(OTS_ERR_INVALID_ARGUMENT, "state field %d is NULL", f);
    ots_status s = copy_field(pl, pl->state[pl->cur][f], state[f], false, pl->geo.padding,
                              pl->geo.padded_size, interior);
    if (s != OTS_OK) return s;
  }
  if (wait) OTS_CUDA(cudaStreamSynchronize(pl->stream), "download");
  return OTS_OK;
}

ots_status ots_download_async(ots_plan* plan, float* const* state) {
  return download_impl(plan, state, false, false);
}

ots_status ots_download_interior_async(ots_plan* plan, float* const* state) {
  return download_impl(plan, state, true, false);
}

ots_status ots_download(ots_plan* plan, float* const* state) {
  return download_impl(plan, state, false);
}

ots_status ots_download_interior(ots_plan* plan, float* const* state) {
  return download_impl(plan, state, true);
}

ots_status ots_plan_device_state(const ots_plan* plan, int32_t field, float** ptr) {
  if (!plan || !ptr || field < 0 || field >= plan->info->ns)
    return fail(OTS_ERR_INVALID_ARGUMENT, "bad state field request");
  *ptr = plan->state[plan->cur][field];
  return OTS_OK;
}

ots_status ots_plan_device_aux(const ots_plan* plan, int32_t field, float** ptr) {
  if (!plan || !ptr || field < 0 || field >= plan->info->na)
    return fail(OTS_ERR_INVALID_ARGUMENT, "bad aux field request");
  *ptr = plan->aux[field];
  return OTS_OK;
}

ots_status ots_plan_set_wait_limit(ots_plan* pl, double seconds) {
  if (!pl) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL plan");
  if (!(seconds > 0.0 && seconds <= 60.0))
    return fail(OTS_ERR_INVALID_ARGUMENT, "wait limit must be in (0, 60] seconds");
  pl->wait_ns = (uint64_t)(seconds * 1e9);
  return OTS_OK;
}

ots_status ots_plan_debug_hold_plane(ots_plan* pl, int32_t plane) {
  if (!pl) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL plan");
  pl->hold_plane = plane < 0 ? -1 : plane;
  return OTS_OK;
}

ots_status ots_plan_enable_clocks(ots_plan* pl, int32_t enable) {
  if (!pl) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL plan");
  OTS_CUDA(cudaSetDevice(pl->device), "cudaSetDevice");
  if (pl->d_clocks) {
    OTS_CUDA(cudaStreamSynchronize(pl->stream), "synchronize");
    cudaFree(pl->d_clocks);
    pl->d_clocks = nullptr;
    pl->clock_warps = 0;
    pl->clocks_valid = false;
  }
  if (!enable) return OTS_OK;
  const int64_t blocks = (int64_t)pl->tile_grid.x * pl->tile_grid.y * pl->tile_grid.z;
  const int64_t threads = (int64_t)pl->tile_block.x * pl->tile_block.y * pl->tile_block.z;
  if (blocks <= 0 || threads <= 0)
    return fail(OTS_ERR_UNSUPPORTED, "clock recording needs the tile kernel's launch shape");
  pl->clock_warps = blocks * ((threads + 31) / 32);
  const size_t bytes = (size_t)pl->clock_warps * ots::kClockWords * sizeof(unsigned);
  OTS_CUDA(cudaMalloc(&pl->d_clocks, bytes), "cudaMalloc clocks");
  OTS_CUDA(cudaMemset(pl->d_clocks, 0, bytes), "cudaMemset clocks");
  return OTS_OK;
}

ots_status ots_plan_clock_records(ots_plan* pl, ots_clock_record* out, int64_t capacity,
                                  int64_t* count) {
  if (!pl || !count) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  if (!pl->d_clocks) return fail(OTS_ERR_INVALID_ARGUMENT, "clock recording is off");
  *count = pl->clocks_valid ? pl->clock_warps : 0;
  if (!pl->clocks_valid || !out || capacity <= 0) return OTS_OK;
  OTS_CUDA(cudaSetDevice(pl->device), "cudaSetDevice");
  std::vector<unsigned> raw((size_t)pl->clock_warps * ots::kClockWords);
  OTS_CUDA(cudaMemcpyAsync(raw.data(), pl->d_clocks, raw.size() * sizeof(unsigned),
                           cudaMemcpyDeviceToHost, pl->stream),
           "read clocks");
  OTS_CUDA(cudaStreamSynchronize(pl->stream), "synchronize");
  const int64_t wpb = ((int64_t)pl->tile_block.x * pl->tile_block.y * pl->tile_block.z + 31) / 32;
  const int64_t n = std::min<int64_t>(capacity, pl->clock_warps);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t blk = i / wpb;
    ots_clock_record& r = out[i];
    r.block_x = (uint32_t)(blk % pl->tile_grid.x);
    r.block_y = (uint32_t)((blk / pl->tile_grid.x) % pl->tile_grid.y);
    r.block_z = (uint32_t)(blk / ((int64_t)pl->tile_grid.x * pl->tile_grid.y));
    r.warp = (uint32_t)(i % wpb);
    r.sm = raw[(size_t)i * ots::kClockWords];
    for (int c = 0; c < 5; ++c) r.clock[c] = raw[(size_t)i * ots::kClockWords + 1 + c];
  }
  return OTS_OK;
}

ots_status ots_plan_stream(const ots_plan* plan, void** s) {
  if (!plan || !s) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  *s = plan->stream;
  return OTS_OK;
}

ots_status ots_host_register(void* ptr, size_t bytes) {
  if (!ptr || !bytes) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL/empty host buffer");
  OTS_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault), "cudaHostRegister");
  return OTS_OK;
}

ots_status ots_host_unregister(void* ptr) {
  if (!ptr) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL host buffer");
  OTS_CUDA(cudaHostUnregister(ptr), "cudaHostUnregister");
  return OTS_OK;
}

ots_status ots_describe(const ots_plan* plan, ots_kv_fn kv, void* user) {
  if (!plan || !kv) return fail(OTS_ERR_INVALID_ARGUMENT, "NULL argument");
  const ots_geometry& g = plan->geo;
  const ots_params& p = plan->prm;
  const StencilInfo& si = *plan->info;
  char v[128];
  auto emit_i = [&](const char* k, long long x) {
    snprintf(v, sizeof v, "%lld", x);
    kv(k, v, user);
  };
  auto emit_d = [&](const char* k, double x) {
    snprintf(v, sizeof v, "%.17g", x);
    kv(k, v, user);
  };
  // printProgramParameters (opencl/common/inc/ProgramGenerator.hpp:19-66)
  const int arrays = si.pp_arrays ? si.pp_arrays : si.ns;
  const int loads = si.pp_loads ? si.pp_loads : (int)(si.r5[0] > 0 ? si.r5[0] : 1);
  const int stores = si.pp_stores ? si.pp_stores : si.ns;
  const int flops = si.pp_flops ? si.pp_flops : (int)si.flops;
  // cells one CTA computes per time level: threads x E for the tile kernel;
  // the whole streamed column (tile x (z segment + pipeline fill)) for the
  // stream kernel
  const bool streamk = g.kernel == OTS_KERNEL_STREAM;
  const int64_t thr = streamk ? (int64_t)g.comps[0] * g.comps[1] * g.comps[2]
                              : (int64_t)p.block_x * (g.dims >= 2 ? p.block_y : 1) *
                                    (g.dims == 3 ? p.block_z : 1) * p.elements_per_thread;
  const int64_t total_fp = thr * p.time_tile * flops;
  int64_t useful = (int64_t)p.time_tile * flops;
  for (int a = 0; a < g.dims; ++a) useful *= std::max(0, g.real_per_block[a]);
  kv("Stencil", si.name, user);
  emit_i("Problem Size", p.problem_size);
  emit_i("Time Tile Size", p.time_tile);
  emit_i("Block Size X", p.block_x);
  emit_i("Block Size Y", g.dims >= 2 ? p.block_y : 1);
  emit_i("Block Size Z", g.dims == 3 ? p.block_z : 1);
  emit_i("Num Blocks X", g.num_blocks[0]);
  emit_i("Num Blocks Y", g.num_blocks[1]);
  emit_i("Num Blocks Z", g.num_blocks[2]);
  emit_i("Elements/Thread", p.elements_per_thread);
  emit_i("Shared Size", (long long)g.shared_size[0] * g.shared_size[1] * g.shared_size[2] * arrays * 4);
  emit_i("Total FP/Block", total_fp);
  emit_i("Useful FP/Block", useful);
  emit_d("Useful Ratio", total_fp ? (double)useful / (double)total_fp : 0.0);
  // the stream kernel reads each cell of its column once (TMA) and writes
  // its interior once
  emit_i("Global Loads/Block", streamk ? thr : thr * loads);
  emit_i("Global Stores/Block", streamk ? useful / std::max<int64_t>(1, (int64_t)p.time_tile * flops)
                                        : thr * stores);
  emit_i("Shared Loads/Block", thr * loads * (p.time_tile - 1));
  emit_i("Shared Stores/Block", thr * stores * (p.time_tile - 1));
  emit_i("Real Per Block X", g.real_per_block[0]);
  emit_i("Real Per Block Y", g.real_per_block[1]);
  if (g.dims == 3) emit_i("Real Per Block Z", g.real_per_block[2]);
  emit_i("Padded Size", g.padded_size);
  emit_i("phase_limit", p.phase_limit);
  emit_i("Time Steps", p.time_steps);
  emit_i("Padding", g.padding);
  emit_i("Real Size", g.real_size);
  emit_i("Register Usage", g.registers);
  static const char* kKernel[] = {"auto", "tile", "stream", "plain", "tex"};
  kv("Kernel", kKernel[(g.kernel >= 0 && g.kernel <= 4) ? g.kernel : 0], user);
  if (g.kernel == OTS_KERNEL_STREAM && (g.dims == 3 || g.dims == 2))
    kv("Stream Arithmetic",
       (g.dims == 3 ? plan->scfg.packed : plan->s2cfg.packed) ? "packed-fp32" : "scalar", user);
  emit_i("Dynamic Shared Bytes", g.shared_bytes);
  kv("Engine", p.engine == OTS_ENGINE_COMPAT ? "compat" : "native", user);
  kv("Variant", p.variant == OTS_VARIANT_REF ? "ref"
                : p.variant == OTS_VARIANT_FAST ? "fast" : "baseline", user);
  if (si.r5[0] >= 0) {
    static const char* kR5[] = {"phase2_global_loads", "phase2_shared_loads", "compute_per_point",
                                "phase3_shared_loads", "phase4_global_stores", "shared_stores",
                                "num_fields", "data_size"};
    for (int i = 0; i < 8; ++i) {
      snprintf(v, sizeof v, "%g", si.r5[i]);
      kv(kR5[i], v, user);
    }
  }
  emit_i("Dimensions", g.dims);
  return OTS_OK;
}

}  // extern "C"
