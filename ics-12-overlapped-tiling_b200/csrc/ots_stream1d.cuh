// ots_stream1d.cuh -- 1D time tile held entirely in registers.
//
// One warp owns a strip of 32 x V consecutive cells (V per lane) plus a halo
// of R T cells per side (rounded up to 4 so every access is a 16-byte
// vector), loads it once, advances it T steps in place -- each step the
// lane's V cells from its own registers, the R cells on either side from the
// neighbouring lanes by shuffle -- and stores the cells that are still valid.
// Each step shrinks the valid region by R cells per side, so T is a runtime
// value: no level rings, no shared memory, no barrier.  Cells outside the
// domain are forced to zero after every step (the Dirichlet ring); the
// update is the op's own apply(), so results are bit-identical to the tile
// and plain kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ots_tile.cuh"

namespace ots {

struct Stream1dParams {
  const float* in;
  float* out;
  int n;          // interior cells
  int T;          // steps of this launch
  int base_step;
  int rpb;        // output cells per warp (multiple of 4)
  int hx;         // halo cells per side (multiple of 4, >= R T)
  int nw;         // warps
  OpArgs op;
};

constexpr int kStream1dThreads = 128;

template <int V, int RX>
struct Row1Acc {
  const float (&c)[V];
  const float (&lh)[RX];  // left lane's last RX cells
  const float (&rh)[RX];  // right lane's first RX cells
  int v, gx, n;
  __device__ __forceinline__ float operator()(int, int, int, int dx) const {
    const int vv = v + dx;
    if (vv < 0) return lh[vv + RX];
    if (vv >= V) return rh[vv - V];
    return c[vv];
  }
  __device__ __forceinline__ bool inside(int, int, int dx) const {
    return (unsigned)(gx + v + dx) < (unsigned)n;
  }
  __device__ __forceinline__ int gy() const { return 0; }
};

// Output cells per warp for cells-per-lane V, radius R and T steps (0 if the
// strip is too narrow).
__host__ __device__ inline int stream1d_rpb(int V, int R, int T, int* hx_out) {
  const int hx = (R * T + 3) / 4 * 4;
  if (hx_out) *hx_out = hx;
  const int r = (32 * V - hx - R * T) / 4 * 4;
  return r >= 4 ? r : 0;
}

template <class Op, int V>
__global__ void __launch_bounds__(kStream1dThreads)
    stream1d_kernel(const __grid_constant__ Stream1dParams p) {
  constexpr int R = Op::RX;
  static_assert(V % 4 == 0 && R <= V, "cells per lane");
  grid_dependency_sync();
  const int w = blockIdx.x * (kStream1dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.nw) return;  // whole warps only
  const int lane = threadIdx.x & 31;
  const int gx = w * p.rpb - p.hx + V * lane;  // multiple of 4
  const int n = p.n;
  unsigned m = 0;  // cells of this lane inside the domain
#pragma unroll
  for (int v = 0; v < V; ++v)
    if ((unsigned)(gx + v) < (unsigned)n) m |= 1u << v;
  const unsigned all = V >= 32 ? 0xFFFFFFFFu : ((1u << V) - 1u);

  float c[V];
  if (m == all) {
#pragma unroll
    for (int j = 0; j < V / 4; ++j) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(p.in + gx) + j);
      c[4 * j] = a.x; c[4 * j + 1] = a.y; c[4 * j + 2] = a.z; c[4 * j + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) c[v] = ((m >> v) & 1) ? __ldg(p.in + gx + v) : 0.0f;
  }

  for (int s = 0; s < p.T; ++s) {
    float lh[R], rh[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      lh[j] = __shfl_up_sync(0xffffffffu, c[V - R + j], 1);
      rh[j] = __shfl_down_sync(0xffffffffu, c[j], 1);
    }
    float nc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const Row1Acc<V, R> acc{c, lh, rh, v, gx, n};
      const float none[1] = {0.0f};
      Op::apply(acc, none, p.op, p.base_step + s, &nc[v]);
    }
    if (m != all) {  // the Dirichlet ring stays zero
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (!((m >> v) & 1)) nc[v] = 0.0f;
    }
#pragma unroll
    for (int v = 0; v < V; ++v) c[v] = nc[v];
  }

  // the cells of this warp's output range [w rpb, (w+1) rpb)
  const int lo = w * p.rpb, hi = lo + p.rpb;
#pragma unroll
  for (int j = 0; j < V / 4; ++j) {
    const int x = gx + 4 * j;
    if (x >= lo && x + 4 <= hi && x + 4 <= n && x >= 0) {
      *(reinterpret_cast<float4*>(p.out + x)) =
          make_float4(c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]);
    } else {
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (x + u >= lo && x + u < hi && (unsigned)(x + u) < (unsigned)n) p.out[x + u] = c[4 * j + u];
    }
  }
}

}  // namespace ots
