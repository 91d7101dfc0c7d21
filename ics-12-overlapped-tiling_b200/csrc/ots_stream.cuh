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
//   * level T writes its plane's interior cells straight to global memory;
//   * a read-only field (Poisson's f) arrives the same way into a second ring
//     of T + 2 planes, one plane ahead of its first use, so every level reads
//     its plane's f from shared memory.
//
// Every mbarrier wait is bounded (p.wait_ns, 2 s unless the host sets it);
// on timeout the CTA records an error word, waits (bounded by time only)
// for its own copies still in flight, and all its threads leave together
// (the host reports OTS_ERR_TIMEOUT).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ots_tile.cuh"

namespace ots {

struct StreamParams {
  CUtensorMap amap;  // the aux field, same box as the state (ops with NA > 0)
  float* out;
  const float* aux;  // star stencils use at most one aux field (Poisson f)
  Layout L;
  int ntx, nty;      // x/y tiles
  int64_t work;      // total output tile-planes = ntx * nty * n2
  int64_t chunk;     // persistent mode: tile-planes per CTA (the last gets fewer)
  int zseg;          // grid mode (> 0): blockIdx.x = tile, blockIdx.y = z segment (x cy)
  int cy;            // CTAs per cluster along y (grid mode); 0 or 1 = no cluster
  int base_step;     // global step index of this launch's first level
  int* err;          // device error word (bit 0: mbarrier wait timed out)
  uint64_t wait_ns;  // limit of every bounded wait (default kWaitNs)
  int hold_plane;    // test hook: CTA 0 never loads this running plane (-1: off)
  OpArgs op;
};

#ifndef OTS_STREAM_STAGES
#define OTS_STREAM_STAGES 4
#endif
constexpr int kStreamStages = OTS_STREAM_STAGES;  // ring depth (power of 2); lookahead = stages - 2
constexpr unsigned kWaitLimit = 1u << 24;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: default limit of a bounded wait

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

// Bounded wait: false if the phase did not complete within `limit_ns` of
// wall time, within kWaitLimit polls, or once another CTA has raised the
// error word (then every CTA stops waiting soon after the first failure).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  const int* err, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255) {
      if (global_ns() - t0 > limit_ns) return false;
      if (*(volatile const int*)err != 0) return false;
    }
  }
  return false;
}

// Drain wait of a failing CTA for one of its own copies still in flight:
// bounded by time and polls only, never cut short by the error word (the
// CTA raised it itself), so the CTA leaves only once the copy has landed or
// the limit has passed.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* bar, unsigned parity,
                                                uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned i = 0; i < kWaitLimit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && global_ns() - t0 > limit_ns) return false;
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

// ---- thread-block cluster helpers (distributed shared memory) ----------
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// shared::cluster address of the same shared location in CTA `rank`
__device__ __forceinline__ uint32_t map_shared(const void* p, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

// Asynchronous 16-byte store into another CTA's shared memory; its bytes
// count against the transaction count of that CTA's mbarrier (the consumer
// arms the barrier with the bytes it expects and waits on it like on a TMA
// copy; no fence on the producer side).
__device__ __forceinline__ void st_async_v4(uint32_t addr, uint32_t bar, float a, float b,
                                            float c, float d) {
  asm volatile(
      "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];"
      ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d), "r"(bar)
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

// Cluster halo rows: 3 rotating slots x T levels x (row from the CTA above,
// row from the CTA below) x TX cells; only clustered launches carry them.
constexpr int kHaloSlots = 3;
__host__ __device__ inline int stream_halo_floats(int T, int TX, int cy) {
  return cy > 1 ? kHaloSlots * T * 2 * TX : 0;
}

// Planes of the aux ring: level t reads f of plane k - t (t = 1..T) while
// plane k + 1's copy is in flight.
__host__ __device__ inline int stream_aux_planes(int T) { return T + 2; }

// Shared bytes: ring + (T-1) double-buffered exchange planes + cluster halo
// rows + aux ring (na > 0) + mbarriers (ring stages, one per halo slot and
// level, one per aux plane).
__host__ __device__ inline size_t stream_smem_bytes(int T, int TX, int TY, int cy = 1,
                                                    int na = 0) {
  size_t plane = (size_t)stream_plane_stride(TX, TY) * sizeof(float);
  const int nf = na > 0 ? stream_aux_planes(T) : 0;
  return (size_t)kStreamStages * plane + (size_t)(T > 1 ? T - 1 : 0) * 2 * plane +
         (size_t)stream_halo_floats(T, TX, cy) * sizeof(float) + (size_t)nf * plane +
         (size_t)(kStreamStages + kHaloSlots * T * 2 + nf) * 8 + 64;
}

// Threads per CTA are capped so that the register rings (3 planes of 4E
// cells per level) stay in registers.
template <int T, int E>
struct StreamThreads {
  static constexpr int kMax = (T * E >= 8) ? 256 : 512;
};

// Packed FP32 pairs cut the issue count but need register pairs; they pay at
// E >= 4 and cost occupancy (more than 128 registers) below that.
template <class Op, int E>
struct StreamPacked {
  static constexpr bool value = Op::PACKED && E >= 4;
};

template <int N>
struct Phase {
  static constexpr int value = N;
};

// blockDim.x (threads along x) must be 8, 16 or 32: a warp then holds whole
// rows of the tile, so every x neighbour a shuffle cannot reach (lane 0's
// left, lane 31's right) is a tile-edge halo cell whose value is never used.
//
// Schedules.  Grid mode (zseg > 0): blockIdx.x = x/y tile, blockIdx.y = z
// segment, so the CTAs resident together stream the same planes of
// neighbouring tiles and their overlapping halo boxes hit in L2.  Persistent
// mode (zseg == 0): one CTA per resident slot, each taking an equal
// contiguous chunk of the (tile, plane) work.  Grid mode is the default: the
// persistent chunks lose the halo reuse in L2.
//
// Clusters along y (CL = true with p.cy > 1, grid mode only): the cy CTAs of a thread-block
// cluster (blockIdx.y = segment * cy + rank) stack their TY-row tiles into one
// tile of cy * TY rows, so the y halo of 2T rows is paid once per cluster, not
// once per CTA.  At every plane each CTA pushes the first and last rows of
// each level (0..T-1) into its neighbours' halo slots with st.async, whose
// bytes complete the transaction count of the neighbour's (slot, level,
// side) mbarrier.  The edge warp that reads a side arms its barriers with the
// bytes it expects and waits (bounded) on them one plane later, right before
// the level that reads the row.  Three rotating slots make the pushes
// race-free: a push into a slot is issued only after the producer's edge
// threads have waited for rows the consumer pushed after it finished reading
// that slot.  The consumer re-arms a slot at the start of plane r for plane
// r+1's pushes (the slot's previous phase was consumed at plane r-1), before
// its own pushes of plane r, which the producer waits for before pushing
// plane r+1: so every arm precedes the bytes it counts.  Plane 0's phase is
// armed before the cluster barrier that opens the kernel.  Clusters need the
// grid schedule (one z segment per CTA).  No pushes happen on a segment's last plane, so
// every push is waited for; a cluster barrier at the start (mbarrier init)
// and at the end (no CTA leaves while a neighbour may still store into it)
// brackets the loop, and every CTA of a cluster runs the same plane count.
template <class Op, int T, int E, bool CL>
__global__ void __launch_bounds__(StreamThreads<T, E>::kMax, 1)
    stream_kernel(const __grid_constant__ CUtensorMap tmap,
                  const __grid_constant__ StreamParams p) {
  constexpr int V = 4;
  constexpr int HX = StreamGeom<T>::HX, HY = StreamGeom<T>::HY;
  constexpr int NST = kStreamStages, LA = kStreamStages - 2;
  constexpr bool FR = Op::NA > 0;                  // aux ring
  constexpr int NF = FR ? T + 2 : 0;               // == stream_aux_planes(T)
  extern __shared__ __align__(128) float smem[];
  const int BX = blockDim.x, BY = blockDim.y;
  const int TX = V * BX, TY = E * BY;
  const int PL = stream_plane_stride(TX, TY);
  const int cy = CL ? (p.cy > 1 ? p.cy : 1) : 1;  // CL=false compiles the cluster code out
  const int crank = cy > 1 ? (int)cluster_rank() : 0;  // == blockIdx.y % cy
  const int rpbx = TX - 2 * HX, rpby = cy * TY - 2 * HY;
  const int tid = threadIdx.x + BX * threadIdx.y;
  const int XB = NST * PL;  // exchange planes start (floats)
  const int HB = XB + (T > 1 ? (T - 1) * 2 * PL : 0);  // cluster halo rows start
  float* const hb = smem + HB;
  const int FB = HB + stream_halo_floats(T, TX, cy);  // aux ring start (128-byte aligned)
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + FB + NF * PL);
  uint64_t* hbars = bars + NST;  // [slot][level][side 0 = row from above, 1 = from below]
  uint64_t* fbars = hbars + (cy > 1 ? kHaloSlots * T * 2 : 0);  // one per aux plane
  const unsigned box_bytes = (unsigned)(TX * TY) * sizeof(float);
  const int n2 = p.L.n2;
  grid_dependency_sync();

  // per-thread constant shared offsets (floats)
  const int lx = V * threadIdx.x, ly = E * threadIdx.y;
  const int o_top = (ly > 0 ? ly - 1 : 0) * TX + lx;          // clamped: tile-edge halo
  const int o_bot = (ly + E < TY ? ly + E : TY - 1) * TX + lx;
  const int o_row0 = ly * TX + lx;
  const bool wx = lx >= HX && lx < HX + rpbx;
  // cluster neighbours: this thread's first row is the CTA's top row (its y-1
  // neighbour lives in the CTA above), its last row the CTA's bottom row
  const bool top_ext = cy > 1 && threadIdx.y == 0 && crank > 0;
  const bool bot_ext = cy > 1 && threadIdx.y == BY - 1 && crank < cy - 1;
  const unsigned row_bytes = (unsigned)TX * sizeof(float);  // one pushed row
  // the first thread of an edge row arms that side's barriers
  const bool arm_top = top_ext && threadIdx.x == 0;
  const bool arm_bot = bot_ext && threadIdx.x == 0;
  // pushes go to the CTA above as its "row from below" (side 1), and to the
  // CTA below as its "row from above" (side 0); remote addresses are mapped
  // at push time (edge threads only) to keep them out of the register budget

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bars[s], 1);
    if (cy > 1)
      for (int s = 0; s < kHaloSlots * T * 2; ++s) mbar_init(&hbars[s], 1);
    for (int s = 0; s < NF; ++s) mbar_init(&fbars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (cy > 1) {
    // plane 0's halo phase (slot 0) is armed before any neighbour can push
    for (int l = 0; l < T; ++l) {
      if (arm_top) mbar_arrive_expect_tx(&hbars[l * 2 + 0], row_bytes);
      if (arm_bot) mbar_arrive_expect_tx(&hbars[l * 2 + 1], row_bytes);
    }
    cluster_sync_all();  // neighbours' barriers exist and are armed before any push
  }

  int64_t pos, pend;
  if (p.zseg > 0) {  // grid mode: neighbouring tiles stream the same planes together
    const int seg = (int)blockIdx.y / cy;
    pos = (int64_t)blockIdx.x * n2 + (int64_t)seg * p.zseg;
    pend = (int64_t)blockIdx.x * n2 + min(n2, (seg + 1) * p.zseg);
  } else {
    pos = (int64_t)blockIdx.x * p.chunk;
    pend = pos + p.chunk < p.work ? pos + p.chunk : p.work;
  }
  int rg = 0;  // running plane counter across segments: ring stage and parity
  int hg = 0;  // running halo-phase counter (pushed planes) across segments
  bool ok = true;
  bool lost = false;  // a halo wait of this thread timed out (reported at the next plane)
  int fail_r = -1;
  while (ok && pos < pend) {
  const int tile = (int)(pos / n2);
  const int zs = (int)(pos - (int64_t)tile * n2);
  const int ze = (int)((pend - pos) < (int64_t)(n2 - zs) ? zs + (pend - pos) : n2);
  pos += ze - zs;
  const int tyi = tile / p.ntx, txi = tile - tyi * p.ntx;
  const int tx0 = txi * rpbx - HX;  // multiple of 4 (TMA x alignment)
  const int ty0 = tyi * rpby - HY + crank * TY;  // this CTA's first row
  const int kb = zs - T, ke = ze + T - 1, nit = ke - kb + 1;
  const int gx = tx0 + lx, gy = ty0 + ly;
  unsigned xyin = 0;
#pragma unroll
  for (int e = 0; e < E; ++e)
#pragma unroll
    for (int v = 0; v < V; ++v)
      if ((unsigned)(gx + v) < (unsigned)p.L.n0 && (unsigned)(gy + e) < (unsigned)p.L.n1)
        xyin |= 1u << (e * V + v);
  const bool xyall = xyin == ((E * V >= 32) ? 0xFFFFFFFFu : ((1u << (E * V)) - 1u));
  float* const obase = p.out + (int64_t)gy * p.L.sy + gx;

  // R[t][slot]: level t's (0 = input) three newest planes of own cells.
  float R[T][3][E][V];
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int e = 0; e < E; ++e)
#pragma unroll
        for (int v = 0; v < V; ++v) R[t][s][e][v] = 0.0f;

  // every thread is past the previous segment's reads of the ring
  __syncthreads();
  // test hook: CTA 0 arms the stage of running plane hold_plane but never
  // loads it, so that plane's wait can only run out (a flag nothing sets)
  const bool hold_cta = p.hold_plane >= 0 && blockIdx.x == 0 && blockIdx.y == 0;
  if (tid == 0) {
    for (int j = 0; j < LA && j < nit; ++j) {
      const int g = rg + j;
      mbar_arrive_expect_tx(&bars[g & (NST - 1)], box_bytes);
      if (!(hold_cta && g == p.hold_plane))
        tma_load_3d(smem + (g & (NST - 1)) * PL, &tmap, tx0, ty0, kb + j, &bars[g & (NST - 1)]);
    }
    if (FR && nit > 1) {  // f of plane kb, first read at iteration 1
      const int fs = rg % (NF > 0 ? NF : 1);
      mbar_arrive_expect_tx(&fbars[fs], box_bytes);
      tma_load_3d(smem + FB + fs * PL, &p.amap, tx0, ty0, kb, &fbars[fs]);
    }
  }

  auto step = [&](auto ph, int r) -> bool {
    constexpr int PH = decltype(ph)::value;
    constexpr int SN = PH, SC = (PH + 2) % 3, SM = (PH + 1) % 3;  // newest, centre, z-1
    const int k = kb + r;
    const int g = rg + r;  // running plane index: ring stage and phase parity
    const int st = g & (NST - 1);
    bool to = !mbar_wait_bounded(&bars[st], (g / NST) & 1, p.err, p.wait_ns);
    if (FR && r >= 1 && !to)  // f of plane k - 1, first read by level 1 now
      to = !mbar_wait_bounded(&fbars[(g - 1) % (NF > 0 ? NF : 1)],
                              ((g - 1) / (NF > 0 ? NF : 1)) & 1, p.err, p.wait_ns);
    // cluster halo: the neighbours' rows of plane r-1 (slot of phase hg+r-1)
    const int hr = (hg + r + kHaloSlots - 1) % kHaloSlots;
    const unsigned hpar = (unsigned)((hg + r - 1) / kHaloSlots) & 1u;
    if (__syncthreads_or(to || lost)) {
      fail_r = g;
      return false;
    }
    // arm the next plane's halo slot: its previous phase (plane r-2) was
    // consumed by this edge warp during plane r-1; the warp's own pushes of
    // this plane follow the arm
    if (cy > 1) {
      if (r + 2 < nit) {
        uint64_t* const hn = &hbars[((hg + r + 1) % kHaloSlots) * T * 2];
        for (int l = 0; l < T; ++l) {
          if (arm_top) mbar_arrive_expect_tx(&hn[l * 2 + 0], row_bytes);
          if (arm_bot) mbar_arrive_expect_tx(&hn[l * 2 + 1], row_bytes);
        }
      }
      __syncwarp();
    }
    if (tid == 0 && r + LA < nit) {
      const int s2 = (g + LA) & (NST - 1);
      mbar_arrive_expect_tx(&bars[s2], box_bytes);
      if (!(hold_cta && g + LA == p.hold_plane))
        tma_load_3d(smem + s2 * PL, &tmap, tx0, ty0, k + LA, &bars[s2]);
    }
    // f of plane k + 1 (read from iteration r + 2 on) into the slot of plane
    // k + 1 - NF = k - T - 1, whose last reader was level T one iteration ago
    if (FR && tid == 0 && r + 2 < nit) {
      const int fs = (g + 1) % (NF > 0 ? NF : 1);
      mbar_arrive_expect_tx(&fbars[fs], box_bytes);
      tma_load_3d(smem + FB + fs * PL, &p.amap, tx0, ty0, k + 1, &fbars[fs]);
    }
    // level 0: the input plane k into registers
    const int pk = st * PL;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float4 a = *reinterpret_cast<const float4*>(smem + pk + o_row0 + e * TX);
      R[0][SN][e][0] = a.x; R[0][SN][e][1] = a.y; R[0][SN][e][2] = a.z; R[0][SN][e][3] = a.w;
    }
    // cluster pushes of this plane (none on the segment's last plane: no
    // neighbour reads them), into slot hw; byte offsets into the remote rows
    const bool push = cy > 1 && r + 1 < nit;
    const int hw = (hg + r) % kHaloSlots;
    float* const hwrow = hb + hw * T * 2 * TX + lx;       // level t at + t*2*TX (+TX: side 1)
    const float* const hrow = hb + hr * T * 2 * TX + lx;  // level t-1 at + (t-1)*2*TX

    const int pc0 = ((g + NST - 1) & (NST - 1)) * PL;   // input plane k-1 (level 1 centre)
    const int xr = XB + ((r - 1) & 1) * PL;              // exchange planes of iteration r-1
    const int xw = XB + (r & 1) * PL;                    // exchange planes of iteration r
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - t;
      const int cp = (t == 1) ? pc0 : xr + (t - 2) * 2 * PL;
      if (r > 0 && !lost) {  // neighbour rows of level t-1, plane r-1
        if (top_ext)
          lost = !mbar_wait_bounded(&hbars[(hr * T + t - 1) * 2 + 0], hpar, p.err, p.wait_ns);
        if (bot_ext && !lost)
          lost = !mbar_wait_bounded(&hbars[(hr * T + t - 1) * 2 + 1], hpar, p.err, p.wait_ns);
      }
      const float* const tp = top_ext ? hrow + (t - 1) * 2 * TX : smem + cp + o_top;
      const float* const bp = bot_ext ? hrow + (t - 1) * 2 * TX + TX : smem + cp + o_bot;
      const float4 tv = *reinterpret_cast<const float4*>(tp);
      const float4 bv = *reinterpret_cast<const float4*>(bp);
      if (t == 1) {
        // level-0 rows of this plane, pushed only after this thread read its
        // slot of plane r-1: a producer that has waited for this push knows
        // the slot it will overwrite next is no longer read
        if (push && top_ext)
          st_async_v4(map_shared(hwrow + TX, crank - 1),
                      map_shared(&hbars[(hw * T) * 2 + 1], crank - 1),
                      R[0][SN][0][0], R[0][SN][0][1], R[0][SN][0][2], R[0][SN][0][3]);
        if (push && bot_ext)
          st_async_v4(map_shared(hwrow, crank + 1), map_shared(&hbars[(hw * T) * 2 + 0], crank + 1),
                      R[0][SN][E - 1][0], R[0][SN][E - 1][1], R[0][SN][E - 1][2],
                      R[0][SN][E - 1][3]);
      }
      float lv[E], rv[E];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        lv[e] = __shfl_up_sync(0xffffffffu, R[t - 1][SC][e][V - 1], 1);
        rv[e] = __shfl_down_sync(0xffffffffu, R[t - 1][SC][e][0], 1);
      }
      const bool zin = (unsigned)q < (unsigned)p.L.n2;
      float fa[E][V];
      if constexpr (FR) {  // f of plane q from the aux ring (zeros outside the domain)
        const float* fp = smem + FB + ((g - t + 16 * NF) % NF) * PL + o_row0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float4 f4 = *reinterpret_cast<const float4*>(fp + e * TX);
          fa[e][0] = f4.x; fa[e][1] = f4.y; fa[e][2] = f4.z; fa[e][3] = f4.w;
        }
      }
      const float tvv[V] = {tv.x, tv.y, tv.z, tv.w};
      const float bvv[V] = {bv.x, bv.y, bv.z, bv.w};
      // level T writes the ring slot of level T-1's oldest plane, which no
      // level needs any more (a scratch slot); levels < T write their own ring
      float (&out)[E][V] = (t < T) ? R[t < T ? t : 0][SN] : R[T - 1][SM];
      if constexpr (StreamPacked<Op, E>::value) {
        // cells (0,1) and (2,3) of each row as packed pairs
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const float(&C)[V] = R[t - 1][SC][e];
          const float* Y0 = e > 0 ? R[t - 1][SC][e - 1] : tvv;
          const float* Y1 = e < E - 1 ? R[t - 1][SC][e + 1] : bvv;
          const float(&M)[V] = R[t - 1][SM][e];
          const float(&N)[V] = R[t - 1][SN][e];
          const float2 mid = make_float2(C[1], C[2]);
          const float2 a = Op::star2(
              make_float2(lv[e], C[0]), make_float2(C[0], C[1]), mid, make_float2(Y0[0], Y0[1]),
              make_float2(Y1[0], Y1[1]), make_float2(M[0], M[1]), make_float2(N[0], N[1]),
              Op::NA > 0 ? make_float2(fa[e][0], fa[e][1]) : make_float2(0.0f, 0.0f), p.op);
          const float2 b = Op::star2(
              mid, make_float2(C[2], C[3]), make_float2(C[3], rv[e]), make_float2(Y0[2], Y0[3]),
              make_float2(Y1[2], Y1[3]), make_float2(M[2], M[3]), make_float2(N[2], N[3]),
              Op::NA > 0 ? make_float2(fa[e][2], fa[e][3]) : make_float2(0.0f, 0.0f), p.op);
          out[e][0] = a.x;
          out[e][1] = a.y;
          out[e][2] = b.x;
          out[e][3] = b.y;
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const float xm = v > 0 ? R[t - 1][SC][e][v - 1] : lv[e];
            const float xp = v < V - 1 ? R[t - 1][SC][e][v + 1] : rv[e];
            const float ym = e > 0 ? R[t - 1][SC][e - 1][v] : tvv[v];
            const float yp = e < E - 1 ? R[t - 1][SC][e + 1][v] : bvv[v];
            out[e][v] = Op::star(xm, R[t - 1][SC][e][v], xp, ym, yp, R[t - 1][SM][e][v],
                                 R[t - 1][SN][e][v], Op::NA > 0 ? fa[e][v] : 0.0f, p.op);
          }
      }
      if (!(zin && xyall)) {  // domain edge: zero the cells outside
#pragma unroll
        for (int e = 0; e < E; ++e)
#pragma unroll
          for (int v = 0; v < V; ++v)
            if (!(zin && ((xyin >> (e * V + v)) & 1))) out[e][v] = 0.0f;
      }
      if (t < T) {
        // other warps need only this thread's first and last rows (y
        // neighbours); x neighbours travel by shuffle
        const int xb = xw + (t - 1) * 2 * PL;
        *reinterpret_cast<float4*>(smem + xb + o_row0) =
            make_float4(out[0][0], out[0][1], out[0][2], out[0][3]);
        if (E > 1)
          *reinterpret_cast<float4*>(smem + xb + o_row0 + (E - 1) * TX) =
              make_float4(out[E - 1][0], out[E - 1][1], out[E - 1][2], out[E - 1][3]);
        if (push && top_ext)
          st_async_v4(map_shared(hwrow + t * 2 * TX + TX, crank - 1),
                      map_shared(&hbars[(hw * T + t) * 2 + 1], crank - 1), out[0][0], out[0][1], out[0][2],
                      out[0][3]);
        if (push && bot_ext)
          st_async_v4(map_shared(hwrow + t * 2 * TX, crank + 1),
                      map_shared(&hbars[(hw * T + t) * 2 + 0], crank + 1), out[E - 1][0], out[E - 1][1],
                      out[E - 1][2], out[E - 1][3]);
      } else if (q >= zs && q < ze && wx) {
        float* dst = obase + (int64_t)q * p.L.sz;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int yy = crank * TY + ly + e;  // row within the (cluster) tile
          if (yy < HY || yy >= HY + rpby) continue;
          const unsigned m = (xyin >> (e * V)) & 0xF;
          if (m == 0xF) {
            *reinterpret_cast<float4*>(dst + (int64_t)e * p.L.sy) =
                make_float4(out[e][0], out[e][1], out[e][2], out[e][3]);
          } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
              if ((m >> v) & 1) dst[(int64_t)e * p.L.sy + v] = out[e][v];
          }
        }
      }
    }
    return true;
  };

  int r = 0;
  for (; r + 2 < nit && ok; r += 3) {
    ok = step(Phase<0>{}, r);
    if (ok) ok = step(Phase<1>{}, r + 1);
    if (ok) ok = step(Phase<2>{}, r + 2);
  }
  if (ok && r < nit) ok = step(Phase<0>{}, r++);
  if (ok && r < nit) ok = step(Phase<1>{}, r++);
  if (ok && cy > 1 && __syncthreads_or(lost)) {  // a halo wait of the last plane timed out
    ok = false;
    fail_r = rg + nit;  // every copy of the segment was consumed: nothing to drain
  }
  if (ok) {
    rg += nit;
    hg += nit - 1;
  }
  if (!ok) {
    if (tid == 0) {
      atomicOr(p.err, 1);
      // drain this CTA's copies still in flight before leaving, each wait
      // bounded by time only: running planes fail_r .. fail_r + LA - 1 were
      // issued
      for (int j = fail_r; j < rg + nit && j < fail_r + LA; ++j)
        mbar_wait_drain(&bars[j & (NST - 1)], (j / NST) & 1, p.wait_ns);
      // aux planes issued but not yet waited for: up to the failing iteration's
      // own plane (issued one iteration before it), from its k - 1 on
      if (FR)
        for (int j = fail_r - 1; j <= fail_r && j < rg + nit - 1; ++j)
          if (j >= rg)
            mbar_wait_drain(&fbars[j % (NF > 0 ? NF : 1)], (j / (NF > 0 ? NF : 1)) & 1,
                            p.wait_ns);
    }
    __syncthreads();
  }
  }  // segments
  // no CTA of a cluster leaves while a neighbour may still push into it: on
  // the normal path every push was waited for; after a failure the pushes
  // already issued land within microseconds, so a failed cluster lingers
  // 20 us past the barrier before its shared memory is released
  if (cy > 1) {
    cluster_sync_all();
    if (!ok) {
      const uint64_t t0 = global_ns();
      while (global_ns() - t0 < 20000ull) {
      }
    }
  }
}

}  // namespace ots
