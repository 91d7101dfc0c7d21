// ots_stream3p.cuh -- z-streamed overlapped time tile for the 3D seven-point
// stencils (Jacobi-3D, and Poisson-3D in its star form) with packed FP32
// arithmetic.
//
// Same scheme and results as stream_kernel (ots_stream.cuh): a CTA owns an
// x/y tile (4 x-cells and E rows per thread, halos of round4(T) columns and T
// rows), walks a z segment plane by plane with all T levels in flight, input
// planes arrive by TMA into a ring of shared stages, x neighbours travel by
// shuffle and y neighbours through shared rows, level T writes its plane
// straight to global memory.  What differs is the arithmetic layout, chosen
// for the sm_100 packed FP32 instructions (add.rn.f32x2 / mul.rn.f32x2: two
// IEEE round-to-nearest operations in one instruction, bit for bit the
// scalar results):
//
//   * a thread's row of 4 cells v0..v3 is held as two 64-bit register pairs,
//     (v0, v2) and (v1, v3).  Every operand of the seven-point sum except two
//     is then a whole pair: the centre, the rows above and below and the
//     planes below and above (same x), and the x neighbour inside the thread
//     ((v1, v3) is the right neighbour of (v0, v2), which is the left
//     neighbour of (v1, v3)).  The two adds that take (v0, v2)'s left
//     neighbours (v-1, v1) or (v1, v3)'s right neighbours (v2, v4) run as
//     scalar adds writing the halves of a pair, so no neighbour pair has to
//     be assembled;
//   * the rows other threads read (a thread's first and last row) go through
//     a compact exchange buffer in this pair order, so they load straight into
//     pairs (ld.shared.v2.b64);
//   * the last level's final multiply is scalar, so its results land in
//     natural x order for one 16-byte store per row.
//
// The rings hold 3 planes per level and 4E cells per plane as pairs: at E=4
// and T=4 that is 192 registers (one CTA of 256 threads per SM), at E=2 96
// (512 threads).  The block shape is a template argument, so every shared
// and exchange offset is an immediate.
//
// The zero Dirichlet ring is applied without a branch: a branch between the
// levels of a plane stops the compiler from overlapping their arithmetic
// (measured: 11-14 % of the kernel's time).  The kernel requires n0 % 4 == 0
// (the host runs the scalar kernel otherwise), so a thread's four x cells are
// all inside the domain or all outside, and a cell is inside exactly when its
// row is inside (y), the thread's columns are (x) and the plane is (z).  Each
// level ANDs the bits of every pair of row e with one 32-bit mask, all ones or
// zero: (plane inside) ? rowmask[e] : 0.  A cleared pair is +0.0 exactly.
//
// Poisson-3D reads its right-hand side f: level t needs f of plane k - t, so
// f streams through a ring of its own (T + 2 planes, TMA, one mbarrier each),
// like the scalar kernel's; its update is (s - h^2 f) / 6 as
// s + (-h^2) f, which is bit for bit s - h^2 f (negation is exact and
// round-to-nearest is symmetric), times 1/6; the product passes through the
// zero-ring AND before the add, so the two never fuse into one rounding.
//
// Every mbarrier wait is bounded (p.wait_ns); on a timeout the CTA records
// the error word, drains its own copies still in flight (bounded by time
// only) and all its threads leave together.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "ots_pair.cuh"
#include "ots_stream.cuh"

namespace ots {

// Block shapes instantiated for the packed kernel: {E, BX, BY}.
struct Shape3p {
  int E, BX, BY;
};
constexpr int kShapes3p = 6;
constexpr Shape3p kShape3p[kShapes3p] = {{4, 16, 16}, {4, 16, 8}, {4, 8, 16},
                                         {2, 16, 32}, {2, 32, 16}, {2, 16, 16}};
inline int shape3p_index(int E, int BX, int BY) {
  for (int i = 0; i < kShapes3p; ++i)
    if (kShape3p[i].E == E && kShape3p[i].BX == BX && kShape3p[i].BY == BY) return i;
  return -1;
}

// Shared layout (floats unless noted; every piece 128-byte aligned):
//   NST ring stages of TX x TY floats (the TMA boxes),
//   exchange rows: levels 1 .. T-1, 2 parities, BY thread rows, 2 rows (the
//   thread row's first and last, pair order), TX floats each,
//   ops with an aux field: T + 2 f stages (TX x TY floats each),
//   NST mbarriers, then one per f stage.
// NST is 8 where that fits the 227 KB a CTA may use, else 4 (and 4 where
// that lets two small CTAs share an SM, below).
constexpr size_t kSmemPerCta = 227 * 1024;
__host__ __device__ constexpr size_t stream3p_stage_floats(int TX, int TY) {
  return (size_t)(TX * TY + 31) / 32 * 32;
}
__host__ __device__ constexpr size_t stream3p_xbuf_floats(int T, int TX, int BY) {
  return (size_t)(T > 1 ? T - 1 : 0) * 2 * BY * 2 * TX;
}
__host__ __device__ constexpr int stream3p_aux_stages(int T, int na) { return na > 0 ? T + 2 : 0; }
__host__ __device__ constexpr size_t stream3p_bytes(int nst, int T, int TX, int TY, int BY,
                                                    int na) {
  return ((size_t)(nst + stream3p_aux_stages(T, na)) * stream3p_stage_floats(TX, TY) +
          stream3p_xbuf_floats(T, TX, BY)) * 4 +
         (size_t)(nst + stream3p_aux_stages(T, na)) * 8;
}
// Blocks of at most 128 threads can run two to an SM (their registers fit
// twice even at 255 a thread): they take the deeper ring only where two CTAs
// still fit the SM's 228 KB (each with the launch's 128 bytes of alignment
// slack and the 1 KB the SM reserves per CTA).  The ring depth barely matters
// (8 stages against 4: within 1 %), occupancy does (Poisson-3D at 16 x 8,
// E = 4, T = 4: one CTA per SM with 8 stages, two with 4).
constexpr size_t kSmemPerSm = 228 * 1024;
__host__ __device__ constexpr bool stream3p_two_fit(size_t bytes) {
  return 2 * (bytes + 128 + 1024) <= kSmemPerSm;
}
__host__ __device__ constexpr int stream3p_stages(int T, int TX, int TY, int BY, int na) {
  return ((TX / 4) * BY <= 128 && !stream3p_two_fit(stream3p_bytes(8, T, TX, TY, BY, na)) &&
          stream3p_two_fit(stream3p_bytes(4, T, TX, TY, BY, na)))
             ? 4
         : stream3p_bytes(8, T, TX, TY, BY, na) <= kSmemPerCta ? 8
                                                              : 4;
}
__host__ __device__ constexpr size_t stream3p_smem_bytes(int T, int TX, int TY, int BY,
                                                         int na) {
  return stream3p_bytes(stream3p_stages(T, TX, TY, BY, na), T, TX, TY, BY, na);
}

// Warps hold whole thread rows (BX = 8, 16 or 32), so the x neighbours a
// shuffle cannot reach are tile-edge halo cells.  Grid: blockIdx.x = x/y
// tile, blockIdx.y = z segment (p.zseg planes).
template <class Op, int T, int E, int BX, int BY>
__global__ void __launch_bounds__(BX * BY, 1)
    stream3p_kernel(const __grid_constant__ CUtensorMap tmap,
                    const __grid_constant__ StreamParams p) {
  constexpr int V = 4;
  constexpr int HX = StreamGeom<T>::HX, HY = StreamGeom<T>::HY;
  constexpr int TX = V * BX, TY = E * BY;
  constexpr bool FR = Op::NA > 0;  // f ring (Poisson-3D)
  constexpr int NF = stream3p_aux_stages(T, Op::NA);
  constexpr int NST = stream3p_stages(T, TX, TY, BY, Op::NA), LA = NST - 2;
  constexpr int PL = (int)stream3p_stage_floats(TX, TY);  // floats per stage
  constexpr int XS = BY * 2 * TX;                          // floats per exchange buffer
  constexpr int rpbx = TX - 2 * HX, rpby = TY - 2 * HY;
  constexpr unsigned box_bytes = (unsigned)(TX * TY) * sizeof(float);
  static_assert(BX == 8 || BX == 16 || BX == 32, "a warp holds whole thread rows");
  static_assert(rpbx >= 4 && rpby >= 1, "the tile keeps an interior");
  static_assert(std::is_same_v<Op, OpJacobi3D> || std::is_same_v<Op, OpPoisson3D>,
                "the packed arithmetic is written for these two ops");
  extern __shared__ __align__(128) float smem[];
  float* const xbase = smem + NST * PL;  // exchange buffers
  float* const fbase = xbase + (T > 1 ? (T - 1) * 2 * XS : 0);  // f stages
  uint64_t* const bars = reinterpret_cast<uint64_t*>(fbase + NF * PL);
  uint64_t* const fbars = bars + NST;
  const int tid = threadIdx.x + BX * threadIdx.y;
  const int n2 = p.L.n2;
  grid_dependency_sync();

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int lx = V * tx, ly = E * ty;
  // shared offsets (floats) of this thread's pieces: its rows in a stage,
  // the rows above / below it in a stage (clamped at the tile edge, where
  // the value is never used), its first / last row and the rows above /
  // below it in an exchange buffer
  const int o_row0 = ly * TX + lx;
  const int o_above = (ly > 0 ? ly - 1 : 0) * TX + lx;
  const int o_below = (ly + E < TY ? ly + E : TY - 1) * TX + lx;
  const int xo_top = (ty * 2 + 0) * TX + lx;
  const int xo_bot = (ty * 2 + 1) * TX + lx;
  const int xo_above = ((ty > 0 ? ty - 1 : ty) * 2 + 1) * TX + lx;
  const int xo_below = ((ty + 1 < BY ? ty + 1 : ty) * 2 + 0) * TX + lx;

  if (tid == 0) {
    for (int s = 0; s < NST + NF; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  const int seg = (int)blockIdx.y;
  const int tile = (int)blockIdx.x;
  const int zs = seg * p.zseg;
  const int ze = min(n2, zs + p.zseg);
  const int tyi = tile / p.ntx, txi = tile - tyi * p.ntx;
  const int tx0 = txi * rpbx - HX;  // multiple of 4 (TMA x alignment)
  const int ty0 = tyi * rpby - HY;
  const int kb = zs - T, nit = (ze - zs) + 2 * T;
  const int gx = tx0 + lx, gy = ty0 + ly;
  // cells of this thread inside the domain in x/y: bit (e * 4 + v)
  unsigned xyin = 0;
#pragma unroll
  for (int e = 0; e < E; ++e)
#pragma unroll
    for (int v = 0; v < V; ++v)
      if ((unsigned)(gx + v) < (unsigned)p.L.n0 && (unsigned)(gy + e) < (unsigned)p.L.n1)
        xyin |= 1u << (e * V + v);
  // per row: all ones if the row's four cells are inside the domain in x/y
  // (n0 % 4 == 0: a thread's columns are all inside or all outside)
  uint32_t rowmask[E];
#pragma unroll
  for (int e = 0; e < E; ++e) rowmask[e] = ((xyin >> (e * V)) & 0xFu) == 0xFu ? ~0u : 0u;
  // level T stores: this thread's columns in the tile interior; rows whose
  // tile row lies in the interior
  const bool st_x = lx >= HX && lx < HX + rpbx && gx < p.L.n0;
  unsigned st_rows = 0;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if (ly + e >= HY && ly + e < HY + rpby && gy + e < p.L.n1) st_rows |= 1u << e;
  const bool st_any = st_x && st_rows != 0;
  const int64_t gsz = p.L.sz, gsy = p.L.sy;
  // level T of iteration r writes plane kb + r - T; the pointer walks one
  // plane per iteration and is dereferenced only for planes in [zs, ze)
  // (where gx, gy and the plane index are all inside the array)
  float* gptr = p.out + (int64_t)gy * gsy + gx + (int64_t)(kb - T) * gsz;
  // Jacobi: coef * sum; Poisson: (sum + (-h^2) f) * (1/6)
  const float coef = FR ? 1.0f / 6.0f : p.op.coef;
  const uint64_t coef2 = p2_make(coef, coef);
  const uint64_t nh2 = p2_make(-p.op.h2, -p.op.h2);
  const int zlo = zs + T, zhi = ze + T;  // iterations' k range whose level-T plane is stored

  // test hook: CTA 0 arms the stage of running plane hold_plane but never
  // loads it, so that plane's wait can only run out (a flag nothing sets)
  const bool hold_cta = p.hold_plane >= 0 && blockIdx.x == 0 && blockIdx.y == 0;
  if (tid == 0) {
    for (int j = 0; j < LA && j < nit; ++j) {
      mbar_arrive_expect_tx(&bars[j], box_bytes);
      if (!(hold_cta && j == p.hold_plane))
        tma_load_3d(smem + j * PL, &tmap, tx0, ty0, kb + j, &bars[j]);
    }
    if (FR && nit > 1) {  // f of plane kb, first read at iteration 1
      mbar_arrive_expect_tx(&fbars[0], box_bytes);
      tma_load_3d(fbase, &p.amap, tx0, ty0, kb, &fbars[0]);
    }
  }

  // R[t][slot][e][pair]: level t's (0 = input) three newest planes
  uint64_t R[T][3][E][2];
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int e = 0; e < E; ++e) R[t][s][e][0] = R[t][s][e][1] = 0ull;

  bool ok = true;
  int fail_r = -1;

  auto step = [&](auto ph, int r) -> bool {
    constexpr int PH = decltype(ph)::value;
    constexpr int SN = PH, SC = (PH + 2) % 3, SM = (PH + 1) % 3;  // newest, centre, z-1
    const int k = kb + r;
    const int st = r & (NST - 1);
    bool to = !mbar_wait_bounded(&bars[st], (r / NST) & 1, p.err, p.wait_ns);
    if (FR && r >= 1 && !to)  // f of plane k - 1, first read by level 1 now
      to = !mbar_wait_bounded(&fbars[(r - 1) % (FR ? NF : 1)], ((r - 1) / (FR ? NF : 1)) & 1,
                              p.err, p.wait_ns);
    if (__syncthreads_or(to)) {
      fail_r = r;
      return false;
    }
    if (tid == 0 && r + LA < nit) {
      const int s2 = (r + LA) & (NST - 1);
      mbar_arrive_expect_tx(&bars[s2], box_bytes);
      if (!(hold_cta && r + LA == p.hold_plane))
        tma_load_3d(smem + s2 * PL, &tmap, tx0, ty0, k + LA, &bars[s2]);
    }
    // f of plane k + 1 (read from iteration r + 2 on) into the stage of plane
    // k + 1 - NF = k - T - 1, whose last reader was level T one iteration ago
    if (FR && tid == 0 && r + 2 < nit) {
      const int fs = (r + 1) % (FR ? NF : 1);
      mbar_arrive_expect_tx(&fbars[fs], box_bytes);
      tma_load_3d(fbase + fs * PL, &p.amap, tx0, ty0, k + 1, &fbars[fs]);
    }
    // level 0: the input plane k into registers (pair order)
    const float* const sk = smem + st * PL + o_row0;
#pragma unroll
    for (int e = 0; e < E; ++e) p2_lds_nat(sk + e * TX, R[0][SN][e][0], R[0][SN][e][1]);
    const float* const pk = smem + ((r + NST - 1) & (NST - 1)) * PL;  // plane k-1
    const int par = r & 1;
    const float* const xr = xbase + (par ^ 1) * XS;  // exchange rows written at r-1
    float* const xw = xbase + par * XS;               // exchange rows written now
    const bool store = st_any && k >= zlo && k < zhi;
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - t;
      uint64_t (&L)[3][E][2] = R[t - 1];
      // rows above / below of level t-1's plane q (other threads' rows)
      uint64_t ab0, ab1, be0, be1;
      if (t == 1) {
        p2_lds_nat(pk + o_above, ab0, ab1);
        p2_lds_nat(pk + o_below, be0, be1);
      } else {
        const float* const xl = xr + (t - 2) * 2 * XS;
        p2_lds(xl + xo_above, ab0, ab1);
        p2_lds(xl + xo_below, be0, be1);
      }
      uint64_t O[E][2];
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const uint64_t c0 = L[SC][e][0], c1 = L[SC][e][1];  // (v0, v2), (v1, v3)
        const float v0 = p2_lo(c0), v2 = p2_hi(c0), v1 = p2_lo(c1), v3 = p2_hi(c1);
        // x neighbours v-1 / v4 from the lanes beside
        const float left = __shfl_up_sync(0xffffffffu, v3, 1);
        const float right = __shfl_down_sync(0xffffffffu, v0, 1);
        const uint64_t ym0 = e > 0 ? L[SC][e > 0 ? e - 1 : 0][0] : ab0;
        const uint64_t ym1 = e > 0 ? L[SC][e > 0 ? e - 1 : 0][1] : ab1;
        const uint64_t yp0 = e < E - 1 ? L[SC][e < E - 1 ? e + 1 : 0][0] : be0;
        const uint64_t yp1 = e < E - 1 ? L[SC][e < E - 1 ? e + 1 : 0][1] : be1;
        // The adds that involve a shuffled neighbour are scalar, written
        // straight into the halves of a new pair; assembling the neighbour
        // pairs (v-1, v1) and (v2, v4) instead would cost register moves.
        uint64_t s0, s1;
        if constexpr (FR) {
          // x-1, x+1, y-1, y+1, z-1, z+1 (OpPoisson3D::star)
          s0 = p2_make(left + v1, v1 + v3);
          s1 = p2_make(v0 + v2, v2 + right);
        } else {
          // x-1, c, x+1, y-1, y+1, z-1, z+1 (opencl/jacobi-3d/jacobi-3d.cpp:282-304)
          s0 = p2_add(p2_make(left + v0, v1 + v2), c1);
          const uint64_t t = p2_add(c0, c1);
          s1 = p2_make(p2_lo(t) + v2, p2_hi(t) + right);
        }
        s0 = p2_add(s0, ym0);
        s1 = p2_add(s1, ym1);
        s0 = p2_add(s0, yp0);
        s1 = p2_add(s1, yp1);
        s0 = p2_add(s0, L[SM][e][0]);
        s1 = p2_add(s1, L[SM][e][1]);
        s0 = p2_add(s0, L[SN][e][0]);
        s1 = p2_add(s1, L[SN][e][1]);
        O[e][0] = s0;
        O[e][1] = s1;
      }
      if constexpr (FR) {  // s + (-h^2) f, f of plane q from its stage
        const float* const fq = fbase + ((r - t + NF) % (FR ? NF : 1)) * PL + o_row0;
        const bool fin = (unsigned)q < (unsigned)n2;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          uint64_t f0, f1;
          p2_lds_nat(fq + e * TX, f0, f1);
          // the product is masked to the domain before the add: besides
          // zeroing it outside, the AND between them keeps the compiler from
          // contracting mul.rn.f32x2 + add.rn.f32x2 into one fused operation
          // (a single rounding; observed as 1-ulp differences in rare cells)
          const uint32_t m = fin ? rowmask[e] : 0u;
          O[e][0] = p2_add(O[e][0], p2_and(p2_mul(nh2, f0), m));
          O[e][1] = p2_add(O[e][1], p2_and(p2_mul(nh2, f1), m));
        }
      }
      if (t < T) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          O[e][0] = p2_mul(coef2, O[e][0]);
          O[e][1] = p2_mul(coef2, O[e][1]);
        }
        // zero ring, branch-free: clear the cells outside the domain
        const bool zin = (unsigned)q < (unsigned)n2;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const uint32_t m = zin ? rowmask[e] : 0u;
          O[e][0] = p2_and(O[e][0], m);
          O[e][1] = p2_and(O[e][1], m);
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
          R[t][SN][e][0] = O[e][0];
          R[t][SN][e][1] = O[e][1];
        }
        // other threads read only this thread's first and last rows
        float* const xl = xw + (t - 1) * 2 * XS;
        p2_sts(xl + xo_top, O[0][0], O[0][1]);
        p2_sts(xl + xo_bot, O[E - 1][0], O[E - 1][1]);
      } else if (store) {
        // level T: final multiply in scalar, natural x order, one store per row
        float4 o[E];
#pragma unroll
        for (int e = 0; e < E; ++e)
          o[e] = make_float4(coef * p2_lo(O[e][0]), coef * p2_lo(O[e][1]),
                             coef * p2_hi(O[e][0]), coef * p2_hi(O[e][1]));
#pragma unroll
        for (int e = 0; e < E; ++e)  // n0 % 4 == 0: four columns, one 16-byte store
          if ((st_rows >> e) & 1u) *reinterpret_cast<float4*>(gptr + e * gsy) = o[e];
      }
    }
    gptr += gsz;
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
  if (!ok) {
    if (tid == 0) {
      atomicOr(p.err, 1);
      // drain this CTA's copies still in flight before leaving, each wait
      // bounded by time only: planes fail_r .. fail_r + LA - 1 were issued
      for (int j = fail_r; j < nit && j < fail_r + LA; ++j)
        mbar_wait_drain(&bars[j & (NST - 1)], (j / NST) & 1, p.wait_ns);
      // f planes issued but not yet waited for: the failing iteration's
      // k - 1 and k (issued one iteration before it)
      if (FR)
        for (int j = fail_r - 1; j <= fail_r && j < nit - 1; ++j)
          if (j >= 0)
            mbar_wait_drain(&fbars[j % (FR ? NF : 1)], (j / (FR ? NF : 1)) & 1, p.wait_ns);
    }
    __syncthreads();
  }
}

}  // namespace ots
