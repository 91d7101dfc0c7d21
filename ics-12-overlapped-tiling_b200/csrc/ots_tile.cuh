// ots_tile.cuh -- overlapped time-tile kernel (all dimensions) and the plain
// one-step-per-launch kernel.
//
// The overlapped tile follows the reference scheme
// (opencl/jacobi-2d/jacobi-2d.cpp:197-514): a CTA of (bx, by, bz) threads,
// each owning E cells along one axis, computes a tile of comps cells, of which
// the inner real_per_block = comps - 2r(T-1) cells per axis are exact after T
// steps and are the only ones written back.  Differences from the reference,
// B200-first:
//   * the whole halo-extended tile (comps + 2r per axis) is loaded once into
//     shared memory with coalesced loads, and T steps run there ping-ponging
//     two shared buffers, one barrier per step (the reference does step 1 from
//     global memory and then two barriers per step);
//   * cells outside the domain read as zero through predicated loads, so the
//     device arrays hold only the interior (no ring), and the problem size
//     need not be a multiple of real_per_block (partial edge tiles);
//   * the write-back respects all axes, including z (the reference ignores
//     writeValidZ, opencl/jacobi-3d/jacobi-3d.cpp:400-405).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "ots_ops.cuh"

namespace ots {

// Programmatic dependent launch.  The launches of one run go out with
// cudaLaunchAttributeProgrammaticStreamSerialization, so launch i+1 can be
// set up and its CTAs scheduled while launch i drains.  Every stencil kernel
// opens with this call, before any global memory access: it lets its own
// successor launch, then waits until its predecessor has completed and that
// launch's writes are visible.  The ping-pong buffers are therefore never
// read or written early; without the attribute both instructions are no-ops.
// Kernels whose grid deliberately fills only part of the GPU (the 2D star
// stream kernel) only wait: an early trigger there lets the successor's CTAs
// be placed while most SMs are idle, and they end up unevenly spread.
__device__ __forceinline__ void grid_dependency_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dependency_sync() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  grid_dependency_wait();
}

// Device layout of one field: x fastest, rows of `sy` floats (sy >= n0,
// 128-byte aligned), planes of `sz` floats.
struct Layout {
  int n0, n1, n2;  // interior extent per axis (1 for unused axes)
  int64_t sy, sz;
};

struct StepParams {
  const float* in[3];
  float* out[3];
  const float* aux[2];
  Layout L;
  int rpb[3];        // interior cells written per CTA and axis
  int T;             // time steps per launch
  int steps;         // total steps of the run
  int base_step;     // global index of this launch's first step
  int phase_limit;   // 0 full, 1/2/3 partial kernels (reference -p)
  OpArgs op;
  // -c: per warp {smid, %clock at entry, after set-up, after the global load
  // and first step, after the in-tile steps, after the write-back}, indexed
  // by linear block x warps per block; nullptr = off
  unsigned* clocks;
  // texture path (the reference's jacobi-2d-tex): state field 0 of the input
  // buffer as a 2D texture with border addressing (0 outside the interior)
  cudaTextureObject_t tex;
};

constexpr int kClockWords = 6;

// Lane 0 of each warp stores its clock record (the reference keeps the
// records of SM 1 only, opencl/jacobi-2d/jacobi-2d.cpp:488-508; all SMs are
// kept here and the host filters).
__device__ __forceinline__ void clock_store(const StepParams& p, int tid, int nth,
                                            const unsigned (&ck)[5]) {
  if (!p.clocks || (tid & 31) != 0) return;
  unsigned sm;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
  const unsigned blk = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  unsigned* r = p.clocks + ((size_t)blk * ((nth + 31) / 32) + (tid >> 5)) * kClockWords;
  r[0] = sm;
#pragma unroll
  for (int i = 0; i < 5; ++i) r[1 + i] = ck[i];
}

__device__ __forceinline__ bool in_domain(const Layout& L, int x, int y, int z) {
  return (unsigned)x < (unsigned)L.n0 && (unsigned)y < (unsigned)L.n1 &&
         (unsigned)z < (unsigned)L.n2;
}

// Accessor over a shared-memory tile (fields `fs` floats apart).
struct SmemAcc {
  const float* p;
  int fs, sy, sz;
  int x, y, z;
  Layout L;
  __device__ __forceinline__ float operator()(int f, int dz, int dy, int dx) const {
    return p[f * fs + dz * sz + dy * sy + dx];
  }
  __device__ __forceinline__ bool inside(int dz, int dy, int dx) const {
    return in_domain(L, x + dx, y + dy, z + dz);
  }
  __device__ __forceinline__ int gy() const { return y; }
};

// Phase-1 values of a two-phase stencil (one float per tile cell, the
// tile's own layout), read at an (dy, dx) offset from the current cell.
struct SmemGAcc {
  const float* p;
  int sy;
  __device__ __forceinline__ float operator()(int dy, int dx) const { return p[dy * sy + dx]; }
};

// Ops that provide TWO_PHASE (phase1 + apply2) run the tile step in two
// phases; every other op keeps its single fused apply().
template <class Op, class = void>
struct TwoPhase {
  static constexpr bool value = false;
};
template <class Op>
struct TwoPhase<Op, std::void_t<decltype(Op::TWO_PHASE)>> {
  static constexpr bool value = Op::TWO_PHASE;
};

// Accessor over global memory with zero outside the domain.
template <int NS>
struct GmemAcc {
  const float* f[NS];
  int64_t i;
  int x, y, z;
  Layout L;
  __device__ __forceinline__ float operator()(int fi, int dz, int dy, int dx) const {
    return inside(dz, dy, dx) ? __ldg(f[fi] + i + dz * L.sz + dy * L.sy + dx) : 0.0f;
  }
  __device__ __forceinline__ bool inside(int dz, int dy, int dx) const {
    return in_domain(L, x + dx, y + dy, z + dz);
  }
  __device__ __forceinline__ int gy() const { return y; }
};

// ------------------------------------------------------------------------
// Overlapped tile: E cells per thread along axis EAX.  E is contiguous per
// thread along y/z (register reuse of the shared neighbours) and strided by
// the block size along x (the reference 1D scheme, jacobi-1d.cpp:249-256,
// which keeps warps on consecutive addresses).
// ------------------------------------------------------------------------
// Threads per CTA shrink as E grows so that the E-cell register blocks do
// not spill; the host rejects larger blocks with OTS_ERR_BLOCK_TOO_LARGE.
template <int E, int NS>
struct TileThreads {
  static constexpr int kMax = (E * NS <= 2) ? 1024 : (E * NS <= 4) ? 512 : 256;
};

// Loads for the tile: through the read-only path in the plain tile kernel;
// at L2 (ld.global.cg) in the batched kernel, whose inputs other CTAs of the
// same launch have just written; through the texture unit in the texture
// variant (state only).
constexpr int kLoadLdg = 0, kLoadCg = 1, kLoadTex = 2;
template <int LD>
__device__ __forceinline__ float tile_load(const float* p) {
  if constexpr (LD == kLoadCg)
    return __ldcg(p);
  else
    return __ldg(p);
}

// One CTA's overlapped time tile.  (bix, biy, biz) is the tile index, (BX,
// BY, BZ) the logical thread block and (tx, ty, tz) this thread in it.
template <class Op, int E, int EAX, int LD>
__device__ __forceinline__ void tile_body(const StepParams& p, int bix, int biy, int biz, int bx,
                                          int by, int bz, int tx, int ty, int tz, float* smem) {
  constexpr int NS = Op::NS, NA = Op::NA;
  constexpr int RX = Op::RX, RY = Op::RY, RZ = Op::RZ;
  const int cx = bx * (EAX == 0 ? E : 1);
  const int cy = by * (EAX == 1 ? E : 1);
  const int cz = bz * (EAX == 2 ? E : 1);
  const int Lx = cx + 2 * RX, Ly = cy + 2 * RY, Lz = cz + 2 * RZ;
  const int LxLy = Lx * Ly, Lvol = LxLy * Lz;
  const int T = p.T;
  // global coordinate of comps cell 0
  const int ox = bix * p.rpb[0] - RX * (T - 1);
  const int oy = biy * p.rpb[1] - RY * (T - 1);
  const int oz = biz * p.rpb[2] - RZ * (T - 1);
  const int tid = tx + bx * (ty + by * tz);
  const int nth = bx * by * bz;
  unsigned ck[5] = {0, 0, 0, 0, 0};
  if (p.clocks) ck[0] = (unsigned)clock();
  if (p.clocks) ck[1] = (unsigned)clock();  // set-up (index arithmetic) done
  if (p.phase_limit == 1) {
    clock_store(p, tid, nth, ck);
    return;
  }

  float* cur = smem;
  float* nxt = smem + NS * Lvol;
  float* gbuf = smem + 2 * NS * Lvol;  // phase-1 values (two-phase ops only)
  if (p.phase_limit != 3) {
    // walk the halo tile with a fixed stride of nth cells, kept as (x, y, z)
    // digits with carries, so no index is divided inside the loop
    const int dz = nth / LxLy, dr = nth - dz * LxLy, dy = dr / Lx, dx = dr - dy * Lx;
    int lz = tid / LxLy, ly = (tid - lz * LxLy) / Lx;
    int lx = tid - lz * LxLy - ly * Lx;
    for (int i = tid; i < Lvol; i += nth) {
      const int gx = ox - RX + lx, gy = oy - RY + ly, gz = oz - RZ + lz;
      const bool in = in_domain(p.L, gx, gy, gz);
      const int64_t gi = (int64_t)gz * p.L.sz + (int64_t)gy * p.L.sy + gx;
#pragma unroll
      for (int f = 0; f < NS; ++f) {
        float v;
        if constexpr (LD == kLoadTex)  // unnormalised texel centres; border mode gives the ring
          v = tex2D<float>(p.tex, (float)gx + 0.5f, (float)gy + 0.5f);
        else
          v = in ? tile_load<LD>(p.in[f] + gi) : 0.0f;
        cur[f * Lvol + i] = v;
        nxt[f * Lvol + i] = v;  // the ring of the second buffer stays defined
      }
      lx += dx;
      ly += dy;
      lz += dz;
      if (lx >= Lx) {  // dx < Lx and dy < Ly: one carry per digit at most
        lx -= Lx;
        ++ly;
      }
      if (ly >= Ly) {
        ly -= Ly;
        ++lz;
      }
    }
  }

  // Owned cells.
  int sidx[E], gxs[E], gys[E], gzs[E];
  bool ins[E];
  float auxv[E][NA > 0 ? NA : 1];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    int lx = tx, ly = ty, lz = tz;
    if (EAX == 0) lx = tx + e * bx;
    if (EAX == 1) ly = ty * E + e;
    if (EAX == 2) lz = tz * E + e;
    sidx[e] = (lz + RZ) * LxLy + (ly + RY) * Lx + (lx + RX);
    gxs[e] = ox + lx;
    gys[e] = oy + ly;
    gzs[e] = oz + lz;
    ins[e] = in_domain(p.L, gxs[e], gys[e], gzs[e]);
    const int64_t gi = (int64_t)gzs[e] * p.L.sz + (int64_t)gys[e] * p.L.sy + gxs[e];
#pragma unroll
    for (int a = 0; a < NA; ++a)
      auxv[e][a] = ins[e] ? tile_load<LD == kLoadTex ? kLoadLdg : LD>(p.aux[a] + gi) : 0.0f;
  }
  __syncthreads();

  int nsteps = p.steps - p.base_step;
  if (nsteps > T) nsteps = T;
  // two-phase ops: phase 1 covers the tile minus G_LO cells at the low and
  // G_HI at the high end of each axis; each thread walks it with a fixed
  // (x, y) stride, so no cell index is divided inside the loop
  int gw = 1, gh = 0, g_dx = 0, g_dy = 0, g_x0 = 0, g_y0 = 0;
  if constexpr (TwoPhase<Op>::value) {
    gw = Lx - Op::G_LO - Op::G_HI;
    gh = Ly - Op::G_LO - Op::G_HI;
    g_dx = nth % gw;
    g_dy = nth / gw;
    g_x0 = tid % gw;
    g_y0 = tid / gw;
  }
  for (int s = 0; s < nsteps; ++s) {
    float res[E][NS];
    if constexpr (TwoPhase<Op>::value) {
      static_assert(Op::DIMS == 2, "two-phase tile step: 2D stencils");
      for (int gx = g_x0, gy = g_y0; gy < gh;) {
        const int lx = Op::G_LO + gx, ly = Op::G_LO + gy;
        const int si = ly * Lx + lx;
        SmemAcc acc{cur + si, Lvol, Lx, LxLy, ox - RX + lx, oy - RY + ly, oz, p.L};
        gbuf[si] = Op::phase1(acc);
        gx += g_dx;
        gy += g_dy;
        if (gx >= gw) {
          gx -= gw;
          ++gy;
        }
      }
      __syncthreads();
#pragma unroll
      for (int e = 0; e < E; ++e) {
        SmemAcc acc{cur + sidx[e], Lvol, Lx, LxLy, gxs[e], gys[e], gzs[e], p.L};
        SmemGAcc gacc{gbuf + sidx[e], Lx};
        Op::apply2(acc, gacc, auxv[e], p.op, p.base_step + s, res[e]);
#pragma unroll
        for (int f = 0; f < NS; ++f)
          if (!ins[e]) res[e][f] = 0.0f;
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        SmemAcc acc{cur + sidx[e], Lvol, Lx, LxLy, gxs[e], gys[e], gzs[e], p.L};
        Op::apply(acc, auxv[e], p.op, p.base_step + s, res[e]);
#pragma unroll
        for (int f = 0; f < NS; ++f)
          if (!ins[e]) res[e][f] = 0.0f;
      }
    }
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int f = 0; f < NS; ++f) nxt[f * Lvol + sidx[e]] = res[e][f];
    __syncthreads();
    float* t = cur;
    cur = nxt;
    nxt = t;
    if (s == 0 && p.clocks) ck[2] = (unsigned)clock();  // global load + first step
    if (p.phase_limit == 2) {
      clock_store(p, tid, nth, ck);
      return;
    }
  }
  if (p.clocks) ck[3] = (unsigned)clock();  // the in-tile steps
  if (p.phase_limit == 3) {
    clock_store(p, tid, nth, ck);
    return;
  }

  // Interior write-back: comps coordinate in [r(T-1), r(T-1) + rpb) per axis.
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int lx = gxs[e] - ox, ly = gys[e] - oy, lz = gzs[e] - oz;
    const bool w = lx >= RX * (T - 1) && lx < RX * (T - 1) + p.rpb[0] && ly >= RY * (T - 1) &&
                   ly < RY * (T - 1) + p.rpb[1] && lz >= RZ * (T - 1) &&
                   lz < RZ * (T - 1) + p.rpb[2];
    if (w && ins[e]) {
      const int64_t gi = (int64_t)gzs[e] * p.L.sz + (int64_t)gys[e] * p.L.sy + gxs[e];
#pragma unroll
      for (int f = 0; f < NS; ++f) p.out[f][gi] = cur[f * Lvol + sidx[e]];
    }
  }
  if (p.clocks) {
    ck[4] = (unsigned)clock();  // write-back
    clock_store(p, tid, nth, ck);
  }
}

template <class Op, int E, int EAX>
__global__ void __launch_bounds__(TileThreads<E, Op::NS>::kMax) tile_kernel(const StepParams p) {
  extern __shared__ float smem[];
  grid_dependency_sync();
  tile_body<Op, E, EAX, kLoadLdg>(p, blockIdx.x, blockIdx.y, blockIdx.z, blockDim.x, blockDim.y,
                                  blockDim.z, threadIdx.x, threadIdx.y, threadIdx.z, smem);
}

// Texture-path variant (opencl/jacobi-2d-tex/jacobi-2d-tex.cpp:235-290): the
// tile's first-step loads come through the texture unit; the in-tile steps
// are the same shared-memory steps.  2D, one state field.
template <class Op, int E>
__global__ void __launch_bounds__(TileThreads<E, Op::NS>::kMax) tile_tex_kernel(const StepParams p) {
  static_assert(Op::DIMS == 2 && Op::NS == 1, "texture path: 2D single-field stencils");
  extern __shared__ float smem[];
  grid_dependency_sync();
  tile_body<Op, E, 1, kLoadTex>(p, blockIdx.x, blockIdx.y, 0, blockDim.x, blockDim.y, 1,
                                threadIdx.x, threadIdx.y, 0, smem);
}

// ------------------------------------------------------------------------
// Plain kernel: one time step per launch, one cell per thread, neighbours
// straight from global memory (L1/L2).  Grid covers the interior exactly.
// ------------------------------------------------------------------------
template <class Op>
__global__ void __launch_bounds__(256) plain_kernel(const StepParams p) {
  constexpr int NS = Op::NS, NA = Op::NA;
  grid_dependency_sync();
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z * blockDim.z + threadIdx.z;
  if (!in_domain(p.L, x, y, z)) return;
  const int64_t i = (int64_t)z * p.L.sz + (int64_t)y * p.L.sy + x;
  float auxv[NA > 0 ? NA : 1];
#pragma unroll
  for (int a = 0; a < NA; ++a) auxv[a] = __ldg(p.aux[a] + i);
  GmemAcc<NS> acc;
#pragma unroll
  for (int f = 0; f < NS; ++f) acc.f[f] = p.in[f];
  acc.i = i;
  acc.x = x;
  acc.y = y;
  acc.z = z;
  acc.L = p.L;
  float res[NS];
  Op::apply(acc, auxv, p.op, p.base_step, res);
#pragma unroll
  for (int f = 0; f < NS; ++f) p.out[f][i] = res[f];
}

}  // namespace ots
