// ots_stream.cuh -- z-streamed overlapped time tile for 3D star stencils.
//
// The reference overlaps time tiles in all three dimensions
// (opencl/jacobi-3d/jacobi-3d.cpp:78-114), which leaves almost no useful
// cells at T > 2 with 3D block shapes.  On B200 the time tile is instead
// overlapped in x/y only and streamed along z: a CTA owns an x/y tile of
// TX x TY cells (4 consecutive x cells and E consecutive y rows per thread)
// and walks a z segment plane by plane with all T time levels in flight.
// Level t works on plane k - t while plane k arrives, so z needs no redundant
// halo (only T planes of pipeline fill per segment).
//
// Data movement per plane:
//   * input planes arrive by TMA (cp.async.bulk.tensor.3d) into a ring of
//     NST shared-memory stages, L = NST - 3 planes ahead, completion tracked
//     by mbarriers; cells outside the domain arrive as zeros (TMA OOB fill),
//     which is the zero Dirichlet ring;
//   * each level keeps its last two planes of own cells in registers (z-1
//     and z neighbours), receives z+1 from the level below in registers, and
//     exchanges x/y neighbours through a double-buffered shared plane per
//     level; one __syncthreads per plane serves every level;
//   * level T writes its plane's interior cells straight to global memory.
//
// Every mbarrier wait is bounded; on timeout the CTA records an error word
// and all its threads leave together (the host reports OTS_ERR_TIMEOUT).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ots_tile.cuh"

namespace ots {

struct StreamParams {
  float* out;
  const float* aux;  // star stencils use at most one aux field (Poisson f)
  Layout L;
  int zseg;          // output planes per CTA along z
  int base_step;     // global step index of this launch's first level
  int* err;          // device error word (bit 0: mbarrier wait timed out)
  OpArgs op;
};

constexpr int kStreamStages = 5;  // ring depth; lookahead = stages - 3
constexpr unsigned kWaitLimit = 1u << 24;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait: false if the phase did not complete within kWaitNs of wall
// time, within kWaitLimit polls, or once another CTA has raised the error
// word (then every CTA stops waiting soon after the first failure).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  const int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255) {
      if (global_ns() - t0 > kWaitNs) return false;
      if (*(volatile const int*)err != 0) return false;
    }
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

template <int T>
struct StreamGeom {
  static constexpr int HX = (T + 3) / 4 * 4;  // x halo rounded to 16 bytes (TMA x alignment)
  static constexpr int HY = T;
};

// Floats between consecutive shared plane buffers: the plane rounded up to
// 128 bytes, because a TMA tensor copy needs a 128-byte aligned shared
// destination (every ring stage is one).
__host__ __device__ inline int stream_plane_stride(int TX, int TY) {
  return (TX * TY + 31) / 32 * 32;
}

// Shared bytes: ring + (T-1) double-buffered exchange planes + mbarriers.
__host__ __device__ inline size_t stream_smem_bytes(int T, int TX, int TY) {
  size_t plane = (size_t)stream_plane_stride(TX, TY) * sizeof(float);
  return (size_t)kStreamStages * plane + (size_t)(T > 1 ? T - 1 : 0) * 2 * plane + 128;
}

// Threads per CTA are capped so that E = 4 (16 cells per thread and level)
// keeps its register rings without spilling.
template <int E>
struct StreamThreads {
  static constexpr int kMax = E >= 4 ? 256 : 512;
};

template <class Op, int T, int E>
__global__ void __launch_bounds__(StreamThreads<E>::kMax, 1)
    stream_kernel(const __grid_constant__ CUtensorMap tmap, const StreamParams p) {
  constexpr int V = 4;
  constexpr int HX = StreamGeom<T>::HX, HY = StreamGeom<T>::HY;
  constexpr int NST = kStreamStages, LA = kStreamStages - 3;
  extern __shared__ __align__(128) float smem[];
  const int BX = blockDim.x, BY = blockDim.y;
  const int TX = V * BX, TY = E * BY;
  const int PL = stream_plane_stride(TX, TY);  // buffer stride; the box is TX*TY
  const int rpbx = TX - 2 * HX, rpby = TY - 2 * HY;
  const int tx0 = blockIdx.x * rpbx - HX;  // multiple of 4
  const int ty0 = blockIdx.y * rpby - HY;
  const int zs = blockIdx.z * p.zseg;
  int ze = zs + p.zseg;
  if (ze > p.L.n2) ze = p.L.n2;
  const int kb = zs - T, ke = ze + T - 1;
  const int tid = threadIdx.x + BX * threadIdx.y;

  float* ring = smem;
  float* xbuf = smem + NST * PL;  // [(T-1)][2][PL]
  uint64_t* bars = reinterpret_cast<uint64_t*>(xbuf + (T > 1 ? (T - 1) * 2 * PL : 0));

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  const unsigned plane_bytes = (unsigned)(TX * TY) * sizeof(float);
  if (tid == 0) {
    for (int j = 0; j < LA && kb + j <= ke; ++j) {
      mbar_arrive_expect_tx(&bars[j % NST], plane_bytes);
      tma_load_3d(ring + (j % NST) * PL, &tmap, tx0, ty0, kb + j, &bars[j % NST]);
    }
  }

  // Own cells: x = 4*tx .. +3, rows y = E*ty .. +E-1 (tile coordinates).
  const int lx = V * threadIdx.x, ly = E * threadIdx.y;
  const int lft = lx > 0 ? lx - 1 : 0;            // clamped: tile-edge cells are halo
  const int rgt = lx + V < TX ? lx + V : TX - 1;
  const int top = ly > 0 ? ly - 1 : 0;
  const int bot = ly + E < TY ? ly + E : TY - 1;
  const int gx = tx0 + lx, gy = ty0 + ly;
  unsigned xyin = 0;  // bit (e*4+v): cell inside the domain in x and y
#pragma unroll
  for (int e = 0; e < E; ++e)
#pragma unroll
    for (int v = 0; v < V; ++v)
      if ((unsigned)(gx + v) < (unsigned)p.L.n0 && (unsigned)(gy + e) < (unsigned)p.L.n1)
        xyin |= 1u << (e * V + v);
  const bool wx = lx >= HX && lx < HX + rpbx;

  float C[T > 1 ? T - 1 : 1][E][V];  // level t (1..T-1): plane k-1-t (centre for level t+1)
  float P[T > 1 ? T - 1 : 1][E][V];  // level t: plane k-2-t
#pragma unroll
  for (int t = 0; t < (T > 1 ? T - 1 : 1); ++t)
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int v = 0; v < V; ++v) C[t][e][v] = P[t][e][v] = 0.0f;

  for (int k = kb; k <= ke; ++k) {
    const int r = k - kb;
    const bool to = !mbar_wait_bounded(&bars[r % NST], (r / NST) & 1, p.err);
    if (__syncthreads_or(to)) {
      if (tid == 0) {
        atomicOr(p.err, 1);
        // drain this CTA's copies still in flight (bounded) before leaving
        for (int j = k; j <= ke && j < k + LA; ++j) {
          const int rj = j - kb;
          mbar_wait_bounded(&bars[rj % NST], (rj / NST) & 1, p.err);
        }
      }
      __syncthreads();
      return;
    }
    if (tid == 0 && k + LA <= ke) {
      const int s = (r + LA) % NST;
      mbar_arrive_expect_tx(&bars[s], plane_bytes);
      tma_load_3d(ring + s * PL, &tmap, tx0, ty0, k + LA, &bars[s]);
    }

    float N[E][V];  // newest plane of the level below, handed upwards
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - t;  // plane this level computes
      // centre plane of level t-1 (its x/y neighbours live in shared memory)
      const float* cp;
      float cen[E][V], zm[E][V], zp[E][V];
      if (t == 1) {
        const float* pk = ring + (r % NST) * PL;            // plane k   (z+1)
        const float* pc = ring + ((r + NST - 1) % NST) * PL;  // plane k-1 (centre)
        const float* pm = ring + ((r + NST - 2) % NST) * PL;  // plane k-2 (z-1)
        cp = pc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float4 a = *reinterpret_cast<const float4*>(pk + (ly + e) * TX + lx);
          const float4 b = *reinterpret_cast<const float4*>(pc + (ly + e) * TX + lx);
          const float4 c = *reinterpret_cast<const float4*>(pm + (ly + e) * TX + lx);
          zp[e][0] = a.x; zp[e][1] = a.y; zp[e][2] = a.z; zp[e][3] = a.w;
          cen[e][0] = b.x; cen[e][1] = b.y; cen[e][2] = b.z; cen[e][3] = b.w;
          zm[e][0] = c.x; zm[e][1] = c.y; zm[e][2] = c.z; zm[e][3] = c.w;
        }
      } else {
        cp = xbuf + ((t - 2) * 2 + ((k - 1) & 1)) * PL;  // written by level t-1 last plane
#pragma unroll
        for (int e = 0; e < E; ++e)
#pragma unroll
          for (int v = 0; v < V; ++v) {
            cen[e][v] = C[t - 2][e][v];
            zm[e][v] = P[t - 2][e][v];
            zp[e][v] = N[e][v];
          }
      }
      float lv[E], rv[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        lv[e] = cp[(ly + e) * TX + lft];
        rv[e] = cp[(ly + e) * TX + rgt];
      }
      const float4 tv = *reinterpret_cast<const float4*>(cp + top * TX + lx);
      const float4 bv = *reinterpret_cast<const float4*>(cp + bot * TX + lx);
      const float tvv[V] = {tv.x, tv.y, tv.z, tv.w};
      const float bvv[V] = {bv.x, bv.y, bv.z, bv.w};
      float fa[E][V];
      if (Op::NA > 0) {
        const bool zin = (unsigned)q < (unsigned)p.L.n2;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const unsigned m = (xyin >> (e * V)) & 0xF;
          const float* src = p.aux + (int64_t)q * p.L.sz + (int64_t)(gy + e) * p.L.sy + gx;
          if (zin && m == 0xF) {
            const float4 f4 = __ldg(reinterpret_cast<const float4*>(src));
            fa[e][0] = f4.x; fa[e][1] = f4.y; fa[e][2] = f4.z; fa[e][3] = f4.w;
          } else {
#pragma unroll
            for (int v = 0; v < V; ++v) fa[e][v] = (zin && ((m >> v) & 1)) ? __ldg(src + v) : 0.0f;
          }
        }
      }
      const bool zin = (unsigned)q < (unsigned)p.L.n2;
      float out[E][V];
#pragma unroll
      for (int e = 0; e < E; ++e)
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const float xm = v > 0 ? cen[e][v - 1] : lv[e];
          const float xp = v < V - 1 ? cen[e][v + 1] : rv[e];
          const float ym = e > 0 ? cen[e - 1][v] : tvv[v];
          const float yp = e < E - 1 ? cen[e + 1][v] : bvv[v];
          float res = Op::star(xm, cen[e][v], xp, ym, yp, zm[e][v], zp[e][v],
                               Op::NA > 0 ? fa[e][v] : 0.0f, p.op);
          const bool in = zin && ((xyin >> (e * V + v)) & 1);
          out[e][v] = in ? res : 0.0f;
        }
      if (t < T) {
        float* xb = xbuf + ((t - 1) * 2 + (k & 1)) * PL;
#pragma unroll
        for (int e = 0; e < E; ++e)
          *reinterpret_cast<float4*>(xb + (ly + e) * TX + lx) =
              make_float4(out[e][0], out[e][1], out[e][2], out[e][3]);
        if (t >= 2) {
          // level t-1's registers have been consumed by this level: shift
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              P[t - 2][e][v] = C[t - 2][e][v];
              C[t - 2][e][v] = N[e][v];
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e)
#pragma unroll
          for (int v = 0; v < V; ++v) N[e][v] = out[e][v];
      } else {
        if (T >= 2) {
#pragma unroll
          for (int e = 0; e < E; ++e)
#pragma unroll
            for (int v = 0; v < V; ++v) {
              P[T - 2][e][v] = C[T - 2][e][v];
              C[T - 2][e][v] = N[e][v];
            }
        }
        if (q >= zs && q < ze && wx) {
#pragma unroll
          for (int e = 0; e < E; ++e) {
            const int yy = ly + e;
            if (yy < HY || yy >= HY + rpby) continue;
            const unsigned m = (xyin >> (e * V)) & 0xF;
            if (m == 0) continue;
            float* dst = p.out + (int64_t)q * p.L.sz + (int64_t)(gy + e) * p.L.sy + gx;
            if (m == 0xF) {
              *reinterpret_cast<float4*>(dst) =
                  make_float4(out[e][0], out[e][1], out[e][2], out[e][3]);
            } else {
#pragma unroll
              for (int v = 0; v < V; ++v)
                if ((m >> v) & 1) dst[v] = out[e][v];
            }
          }
        }
      }
    }
  }
}

}  // namespace ots
