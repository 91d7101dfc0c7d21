// ots_stream2d.cuh -- y-streamed overlapped time tile for 2D star stencils.
//
// The 2D counterpart of the z-streamed kernel: one warp owns an x strip of
// 128 cells (4 consecutive cells per lane) and walks a y segment row by row
// with all T time levels in flight; level t works on row k - t while row k
// arrives.  x is overlapped (a halo of T cells per side, rounded up to 4 so
// every row access is a 16-byte vector), y needs no redundant halo (only the
// 2T-1 rows of pipeline fill per segment).  Each level keeps its three newest
// rows of own cells in registers; x neighbours travel by warp shuffle (lane
// 0's left and lane 31's right are strip-edge halo cells whose values are
// never used).  There is no shared memory and no block-wide barrier: warps
// are independent, and input rows are fetched from global memory (L2 for
// grids that fit it) three rows ahead of use.
//
// Operand order per update is the stencil's own (Op::star2d), so results are
// bit-identical to the tile and plain kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "ots_pair.cuh"
#include "ots_tile.cuh"

namespace ots {

struct Stream2dParams {
  const float* in;
  float* out;
  const float* aux;  // Poisson f, or nullptr
  Layout L;          // n0 = x extent, n1 = y extent, sy = row pitch
  int ntx;           // x strips
  int nseg;          // y segments
  int zseg;          // rows per segment
  int base_step;
  OpArgs op;
};

// Stencils with the five-point form star2d(x-1, c, x+1, y-1, y+1, f).
template <class Op, class = void>
struct HasStar2D : std::false_type {};
template <class Op>
struct HasStar2D<Op, std::void_t<decltype(&Op::star2d)>> : std::true_type {};

constexpr int kStream2dThreads = 128;  // 4 independent warps per CTA
constexpr int kStream2dWidth = 128;    // cells per strip (32 lanes x 4)

__host__ __device__ inline int stream2d_halo(int T) { return (T + 3) / 4 * 4; }

// Rows per y segment for one grid on its own.  Every warp streams one
// segment plus its 2T-row pipeline fill, so all warps take equally long and
// the launch lasts as long as the SM given the most CTAs: ceil(CTAs / SMs)
// of them, run in rounds of at most `warps_per_sm` resident warps, each
// round one warp's iterations, stretched by the issue share once more than
// 12 warps share the SM.  The segment count trades the pipeline fill against
// those rounds; a grid a few CTAs over a whole round pays a second one.
inline int stream2d_zseg(int n, int T, int ntx, int sm_count, int warps_per_sm) {
  constexpr int wpb = kStream2dThreads / 32;
  constexpr double kSatWarps = 12.0;
  const int64_t sms = sm_count > 1 ? sm_count : 1;
  const int64_t bps = warps_per_sm / wpb > 1 ? warps_per_sm / wpb : 1;  // resident CTAs per SM
  const double full_round = wpb * bps > kSatWarps ? wpb * bps / kSatWarps : 1.0;
  double best = 1e300;
  int best_seg = n;
  const int maxseg = n / (T > 1 ? T : 1) > 1 ? n / (T > 1 ? T : 1) : 1;
  for (int nseg = 1; nseg <= maxseg; ++nseg) {
    const int zseg = (n + nseg - 1) / nseg;
    const int segs = (n + zseg - 1) / zseg;
    const double len = zseg + 2.0 * T;
    const int64_t ctas = ((int64_t)ntx * segs + wpb - 1) / wpb;
    const int64_t per_sm = (ctas + sms - 1) / sms;
    const int64_t rem = per_sm % bps;
    const double last = wpb * rem > kSatWarps ? wpb * rem / kSatWarps : 1.0;
    const double cost = len * ((double)(per_sm / bps) * full_round + (rem ? last : 0.0));
    if (cost < best * 0.999) {
      best = cost;
      best_seg = zseg;
    }
  }
  return best_seg;
}

template <int N>
struct Phase2 {
  static constexpr int value = N;
};

// Row loads: through the read-only path (standalone kernel) or at L2 (the
// batched kernel, whose inputs other SMs have just written).
template <int LD>
__device__ __forceinline__ float4 s2_load4(const float* p) {
  if constexpr (LD == kLoadCg)
    return __ldcg(reinterpret_cast<const float4*>(p));
  else
    return __ldg(reinterpret_cast<const float4*>(p));
}
template <int LD>
__device__ __forceinline__ float s2_load1(const float* p) {
  if constexpr (LD == kLoadCg)
    return __ldcg(p);
  else
    return __ldg(p);
}

// One warp's strip x segment: the whole time tile of T levels.  Called by
// all 32 lanes of a warp together (shuffles).
template <class Op, int T, int LD>
__device__ __forceinline__ void stream2d_body(const Stream2dParams& p, int strip, int seg) {
  constexpr int V = 4;
  constexpr int HX = (T + 3) / 4 * 4;
  constexpr int RPBX = kStream2dWidth - 2 * HX;
  const int lane = threadIdx.x & 31;
  const int nx = p.L.n0, ny = p.L.n1;
  const int64_t sy = p.L.sy;
  const int tx0 = strip * RPBX - HX;  // multiple of 4
  const int lx = V * lane;
  const int gx = tx0 + lx;
  unsigned xin = 0;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if ((unsigned)(gx + v) < (unsigned)nx) xin |= 1u << v;
  const bool xall = xin == 0xFu;
  const bool wx = lx >= HX && lx < HX + RPBX;  // this lane's cells are output columns
  const int ys = seg * p.zseg;
  const int ye = min(ny, ys + p.zseg);
  const int kb = ys - T;
  const int nit = (ye + T - 1) - kb + 1;

  // one input row (zeros outside the domain)
  auto load_row = [&](int k, float (&d)[V]) {
#pragma unroll
    for (int v = 0; v < V; ++v) d[v] = 0.0f;
    if ((unsigned)k < (unsigned)ny) {
      const float* src = p.in + (int64_t)k * sy + gx;
      if (xall) {
        const float4 a = s2_load4<LD>(src);
        d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if ((xin >> v) & 1) d[v] = s2_load1<LD>(src + v);
      }
    }
  };

  float R[T][3][V];  // level t (0 = input): three newest rows of own cells
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
      for (int v = 0; v < V; ++v) R[t][s][v] = 0.0f;
  float P[3][V];  // prefetched input rows k .. k+2
#pragma unroll
  for (int j = 0; j < 3; ++j) load_row(kb + j, P[j]);

  auto step = [&](auto ph, int r) {
    constexpr int PH = decltype(ph)::value;
    constexpr int SN = PH, SC = (PH + 2) % 3, SM = (PH + 1) % 3;  // newest, centre, y-1
    const int k = kb + r;
    // level 0: the prefetched row k; its slot takes row k + 3
#pragma unroll
    for (int v = 0; v < V; ++v) R[0][SN][v] = P[PH][v];
    load_row(k + 3, P[PH]);
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - t;
      const float(&C)[V] = R[t - 1][SC];
      const float(&M)[V] = R[t - 1][SM];
      const float(&N)[V] = R[t - 1][SN];
      const float lv = __shfl_up_sync(0xffffffffu, C[V - 1], 1);
      const float rv = __shfl_down_sync(0xffffffffu, C[0], 1);
      const bool qin = (unsigned)q < (unsigned)ny;
      float f[V] = {0.0f, 0.0f, 0.0f, 0.0f};
      if (Op::NA > 0 && qin) {
        const float* src = p.aux + (int64_t)q * sy + gx;
        if (xall) {
          const float4 a = s2_load4<kLoadLdg>(src);  // read-only for the whole run
          f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if ((xin >> v) & 1) f[v] = s2_load1<kLoadLdg>(src + v);
        }
      }
      // level T writes the slot of level T-1's oldest row, which no level
      // needs any more; each cell reads M[v] before its own out[v] is written
      float(&out)[V] = (t < T) ? R[t < T ? t : 0][SN] : R[T - 1][SM];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const float xm = v > 0 ? C[v - 1] : lv;
        const float xp = v < V - 1 ? C[v + 1] : rv;
        out[v] = Op::star2d(xm, C[v], xp, M[v], N[v], f[v], p.op);
      }
      if (!(qin && xall)) {  // domain edge: the Dirichlet ring stays zero
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (!(qin && ((xin >> v) & 1))) out[v] = 0.0f;
      }
      if (t == T && q >= ys && q < ye && wx) {
        float* dst = p.out + (int64_t)q * sy + gx;
        if (xall) {
          *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if ((xin >> v) & 1) dst[v] = out[v];
        }
      }
    }
  };

  int r = 0;
  for (; r + 2 < nit; r += 3) {
    step(Phase2<0>{}, r);
    step(Phase2<1>{}, r + 1);
    step(Phase2<2>{}, r + 2);
  }
  if (r < nit) step(Phase2<0>{}, r++);
  if (r < nit) step(Phase2<1>{}, r++);
}

template <class Op, int T>
__global__ void __launch_bounds__(kStream2dThreads)
    stream2d_kernel(const __grid_constant__ Stream2dParams p) {
  grid_dependency_wait();  // no early trigger: see grid_dependency_sync
  const int w = blockIdx.x * (kStream2dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.ntx * p.nseg) return;  // whole warps only
  stream2d_body<Op, T, kLoadLdg>(p, w % p.ntx, w / p.ntx);
}

// ------------------------------------------------------------------------
// The same y-streamed scheme with packed FP32 arithmetic, for the two
// five-point stencils whose update is adds and multiplies only (Jacobi-2D;
// Poisson-2D with its right-hand side).  A lane's four cells v0..v3 are held
// as the pairs (v0, v2) and (v1, v3) in 64-bit registers, as in the packed 3D
// kernel (ots_stream3p.cuh): each add.rn.f32x2 / mul.rn.f32x2 does two IEEE
// operations, bit for bit the scalar ones, in the op's operand order; the
// adds that take a shuffled x neighbour (v-1 or v4) run scalar into the halves
// of a new pair.  The zero ring is one 32-bit AND per pair half and level --
// and that AND between a level's multiply and the next level's adds also
// keeps the two from being fused into one rounding.  With n0 % 4 == 0 a
// lane's four cells are all inside the domain or all outside, so one mask
// serves both halves; otherwise (EDGE) each half has its own, the edge lane's
// input cells beyond n0 are cleared on load and its cells are stored one by
// one.  Level T's multiply is scalar, so its results land in natural x order
// for one 16-byte store.
template <class Op>
struct Packed2D
    : std::bool_constant<std::is_same_v<Op, OpJacobi2D> || std::is_same_v<Op, OpPoisson2D>> {};

template <class Op, int T, int LD, bool EDGE>
__device__ __forceinline__ void stream2dp_body(const Stream2dParams& p, int strip, int seg) {
  static_assert(Packed2D<Op>::value, "packed form written for Jacobi-2D and Poisson-2D");
  constexpr bool PO = std::is_same_v<Op, OpPoisson2D>;
  constexpr int V = 4;
  constexpr int HX = (T + 3) / 4 * 4;
  constexpr int RPBX = kStream2dWidth - 2 * HX;
  const int lane = threadIdx.x & 31;
  const int ny = p.L.n1;
  const int64_t sy = p.L.sy;
  const int gx = strip * RPBX - HX + V * lane;  // multiple of 4
  // the lane's cells inside the domain in x: v < kx (all four, or none,
  // when n0 % 4 == 0); a lane left of the domain (gx < 0, a multiple of 4)
  // has none
  const int kx = gx < 0 ? 0 : p.L.n0 - gx;
  const bool xin = kx > 0;
  const bool xfull = kx >= 4;
  // per pair half: (v0, v2) and (v1, v3)
  const uint32_t mx00 = kx > 0 ? ~0u : 0u, mx02 = kx > 2 ? ~0u : 0u;
  const uint32_t mx11 = kx > 1 ? ~0u : 0u, mx13 = kx > 3 ? ~0u : 0u;
  const bool wx = V * lane >= HX && V * lane < HX + RPBX;
  const int ys = seg * p.zseg;
  const int ye = min(ny, ys + p.zseg);
  const int kb = ys - T;
  const int nit = (ye + T - 1) - kb + 1;
  // Jacobi: coef * sum; Poisson: (sum + (-h^2) f) * 0.25
  const float coef = PO ? 0.25f : p.op.coef;
  const uint64_t coef2 = p2_make(coef, coef);
  const uint64_t nh2 = p2_make(-p.op.h2, -p.op.h2);

  // one row of four cells as the pairs (v0, v2), (v1, v3); zeros outside
  auto load_pairs = [&](const float* base, int k, uint64_t& a0, uint64_t& a1, auto ld) {
    a0 = a1 = 0ull;
    if (xin && (unsigned)k < (unsigned)ny) {
      const float4* src = reinterpret_cast<const float4*>(base + (int64_t)k * sy + gx);
      const float4 a = decltype(ld)::value == kLoadCg ? __ldcg(src) : __ldg(src);
      a0 = p2_make(a.x, a.z);
      a1 = p2_make(a.y, a.w);
      if constexpr (EDGE) {  // cells beyond n0 (the row's padding) read as zero
        a0 = p2_and2(a0, mx00, mx02);
        a1 = p2_and2(a1, mx11, mx13);
      }
    }
  };
  using LdIn = std::integral_constant<int, LD>;
  using LdRo = std::integral_constant<int, kLoadLdg>;  // f: read-only for the whole run

  uint64_t R[T][3][2];  // level t (0 = input): three newest rows, as pairs
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int s = 0; s < 3; ++s) R[t][s][0] = R[t][s][1] = 0ull;
  uint64_t P[3][2];  // prefetched input rows k .. k+2
#pragma unroll
  for (int j = 0; j < 3; ++j) load_pairs(p.in, kb + j, P[j][0], P[j][1], LdIn{});
  // Poisson: level t's f row of the coming iteration, fetched one iteration
  // ahead (a load issued where it is used stalls the level on L2)
  uint64_t Fq[PO ? T : 1][2];
  if constexpr (PO) {
#pragma unroll
    for (int t = 1; t <= T; ++t) load_pairs(p.aux, kb - t, Fq[t - 1][0], Fq[t - 1][1], LdRo{});
  }

  auto step = [&](auto ph, int r) {
    constexpr int PH = decltype(ph)::value;
    constexpr int SN = PH, SC = (PH + 2) % 3, SM = (PH + 1) % 3;  // newest, centre, y-1
    const int k = kb + r;
    R[0][SN][0] = P[PH][0];
    R[0][SN][1] = P[PH][1];
    load_pairs(p.in, k + 3, P[PH][0], P[PH][1], LdIn{});
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - t;
      const uint64_t c0 = R[t - 1][SC][0], c1 = R[t - 1][SC][1];
      const uint64_t m0 = R[t - 1][SM][0], m1 = R[t - 1][SM][1];  // row y-1
      const uint64_t n0 = R[t - 1][SN][0], n1 = R[t - 1][SN][1];  // row y+1
      const float v0 = p2_lo(c0), v2 = p2_hi(c0), v1 = p2_lo(c1);
      const float left = __shfl_up_sync(0xffffffffu, p2_hi(c1), 1);  // v-1
      const float right = __shfl_down_sync(0xffffffffu, v0, 1);      // v4
      uint64_t s0, s1;
      if constexpr (PO) {
        // y-1, x-1, x+1, y+1 (OpPoisson2D::star2d)
        s0 = p2_add(p2_make(p2_lo(m0) + left, p2_hi(m0) + v1), c1);
        s0 = p2_add(s0, n0);
        const uint64_t u = p2_add(m1, c0);
        s1 = p2_add(p2_make(p2_lo(u) + v2, p2_hi(u) + right), n1);
      } else {
        // x-1, c, x+1, y-1, y+1 (OpJacobi2D::star2d)
        s0 = p2_add(p2_make(left + v0, v1 + v2), c1);
        const uint64_t u = p2_add(c0, c1);
        s1 = p2_make(p2_lo(u) + v2, p2_hi(u) + right);
        s0 = p2_add(p2_add(s0, m0), n0);
        s1 = p2_add(p2_add(s1, m1), n1);
      }
      const bool qin = (unsigned)q < (unsigned)ny;
      const uint32_t mq = qin ? ~0u : 0u;
      // the zero-ring masks of this level: (v0, v2) and (v1, v3)
      const uint32_t m00 = EDGE ? (mq & mx00) : (mq & mx13), m02 = EDGE ? (mq & mx02) : m00;
      const uint32_t m11 = EDGE ? (mq & mx11) : m00, m13 = EDGE ? (mq & mx13) : m00;
      if constexpr (PO) {  // s + (-h^2) f, the product masked before the add
        s0 = p2_add(s0, p2_and2(p2_mul(nh2, Fq[t - 1][0]), m00, m02));
        s1 = p2_add(s1, p2_and2(p2_mul(nh2, Fq[t - 1][1]), m11, m13));
        load_pairs(p.aux, q + 1, Fq[t - 1][0], Fq[t - 1][1], LdRo{});
      }
      if (t < T) {
        R[t][SN][0] = p2_and2(p2_mul(coef2, s0), m00, m02);
        R[t][SN][1] = p2_and2(p2_mul(coef2, s1), m11, m13);
      } else if (q >= ys && q < ye && wx && xin) {
        const float4 o =
            make_float4(coef * p2_lo(s0), coef * p2_lo(s1), coef * p2_hi(s0), coef * p2_hi(s1));
        float* const dst = p.out + (int64_t)q * sy + gx;
        if (!EDGE || xfull) {
          *reinterpret_cast<float4*>(dst) = o;
        } else {  // the edge lane: its cells inside the domain only
          dst[0] = o.x;
          if (kx > 1) dst[1] = o.y;
          if (kx > 2) dst[2] = o.z;
        }
      }
    }
  };

  int r = 0;
  for (; r + 2 < nit; r += 3) {
    step(Phase2<0>{}, r);
    step(Phase2<1>{}, r + 1);
    step(Phase2<2>{}, r + 2);
  }
  if (r < nit) step(Phase2<0>{}, r++);
  if (r < nit) step(Phase2<1>{}, r++);
}

template <class Op, int T>
__global__ void __launch_bounds__(kStream2dThreads)
    stream2dp_kernel(const __grid_constant__ Stream2dParams p) {
  grid_dependency_wait();  // no early trigger: see grid_dependency_sync
  const int w = blockIdx.x * (kStream2dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.ntx * p.nseg) return;  // whole warps only
  if (p.L.n0 % 4 == 0)
    stream2dp_body<Op, T, kLoadLdg, false>(p, w % p.ntx, w / p.ntx);
  else
    stream2dp_body<Op, T, kLoadLdg, true>(p, w % p.ntx, w / p.ntx);
}

// ------------------------------------------------------------------------
// Generic y-streamed kernel: any 2D stencil, through the op's own apply().
//
// Radius R = Op::RY rows: level t works on row k - R t, and each level keeps
// its 2R+1 newest rows of every state field in registers.  The op reads its
// neighbourhood through RingAcc, which maps (field, dy, dx) onto those rows
// at compile time; cells up to RX = Op::RX to the left/right of a lane's
// four come from the neighbouring lanes (shuffled once per row and level).
// Aux fields are read at the cell only (every 2D op here does).  The x halo
// is R T rounded up to 4, so strips hold 128 - 2 roundup4(R T) output cells.
// ------------------------------------------------------------------------
struct Stream2dgParams {
  const float* in[3];
  float* out[3];
  const float* aux[2];
  Layout L;
  int ntx, nseg, zseg, base_step;
  OpArgs op;
};

template <int NS, int D, int RX, int PH, int R>
struct RingAcc {
  static constexpr int V = 4;
  const float (&ring)[NS][D][V];
  const float (&lh)[NS][D][RX];  // left lane's last RX cells of each row
  const float (&rh)[NS][D][RX];  // right lane's first RX cells
  int v, gx, q, nx, ny;
  __device__ __forceinline__ float operator()(int f, int, int dy, int dx) const {
    const int s = (PH + dy - R + 2 * D) % D;  // row q + dy of the previous level
    const int vv = v + dx;
    if (vv < 0) return lh[f][s][vv + RX];
    if (vv >= V) return rh[f][s][vv - V];
    return ring[f][s][vv];
  }
  __device__ __forceinline__ bool inside(int, int dy, int dx) const {
    return (unsigned)(gx + v + dx) < (unsigned)nx && (unsigned)(q + dy) < (unsigned)ny;
  }
  __device__ __forceinline__ int gy() const { return q; }
};

template <int N>
struct PhaseG {
  static constexpr int value = N;
};

template <class Op, int T>
__global__ void __launch_bounds__(kStream2dThreads)
    stream2dg_kernel(const __grid_constant__ Stream2dgParams p) {
  constexpr int V = 4, NS = Op::NS, NA = Op::NA, R = Op::RY, RX = Op::RX, D = 2 * R + 1;
  constexpr int HX = (R * T + 3) / 4 * 4;
  constexpr int RPBX = kStream2dWidth - 2 * HX;
  static_assert(RX <= V && RPBX >= 4, "stencil reach / depth");
  grid_dependency_sync();
  const int w = blockIdx.x * (kStream2dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.ntx * p.nseg) return;  // whole warps only
  const int strip = w % p.ntx, seg = w / p.ntx;
  const int lane = threadIdx.x & 31;
  const int nx = p.L.n0, ny = p.L.n1;
  const int64_t sy = p.L.sy;
  const int gx = strip * RPBX - HX + V * lane;  // multiple of 4
  unsigned xin = 0;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if ((unsigned)(gx + v) < (unsigned)nx) xin |= 1u << v;
  const bool xall = xin == 0xFu;
  const bool wx = V * lane >= HX && V * lane < HX + RPBX;
  const int ys = seg * p.zseg;
  const int ye = min(ny, ys + p.zseg);
  const int kb = ys - R * T;
  const int nit = (ye + R * T - 1) - kb + 1;

  auto load4 = [&](const float* base, int k, float (&d)[V]) {
#pragma unroll
    for (int v = 0; v < V; ++v) d[v] = 0.0f;
    if ((unsigned)k < (unsigned)ny) {
      const float* src = base + (int64_t)k * sy + gx;
      if (xall) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(src));
        d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if ((xin >> v) & 1) d[v] = __ldg(src + v);
      }
    }
  };

  float Rg[T][NS][D][V];  // level t (0 = input): 2R+1 newest rows of every field
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int f = 0; f < NS; ++f)
#pragma unroll
      for (int s = 0; s < D; ++s)
#pragma unroll
        for (int v = 0; v < V; ++v) Rg[t][f][s][v] = 0.0f;
  float P[D][NS][V];  // input rows k .. k + D - 1, fetched ahead
#pragma unroll
  for (int j = 0; j < D; ++j)
#pragma unroll
    for (int f = 0; f < NS; ++f) load4(p.in[f], kb + j, P[j][f]);

  auto step = [&](auto ph, int r) {
    constexpr int PH = decltype(ph)::value;  // slot of the newest row
    const int k = kb + r;
#pragma unroll
    for (int f = 0; f < NS; ++f) {
#pragma unroll
      for (int v = 0; v < V; ++v) Rg[0][f][PH][v] = P[PH][f][v];
      load4(p.in[f], k + D, P[PH][f]);
    }
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - R * t;
      float lh[NS][D][RX], rh[NS][D][RX];
#pragma unroll
      for (int f = 0; f < NS; ++f)
#pragma unroll
        for (int s = 0; s < D; ++s)
#pragma unroll
          for (int j = 0; j < RX; ++j) {
            lh[f][s][j] = __shfl_up_sync(0xffffffffu, Rg[t - 1][f][s][V - RX + j], 1);
            rh[f][s][j] = __shfl_down_sync(0xffffffffu, Rg[t - 1][f][s][j], 1);
          }
      const bool qin = (unsigned)q < (unsigned)ny;
      float res[V][NS];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        float av[NA > 0 ? NA : 1];
#pragma unroll
        for (int a = 0; a < NA; ++a)
          av[a] = (qin && ((xin >> v) & 1)) ? __ldg(p.aux[a] + (int64_t)q * sy + gx + v) : 0.0f;
        const RingAcc<NS, D, RX, PH, R> acc{Rg[t - 1], lh, rh, v, gx, q, nx, ny};
        Op::apply(acc, av, p.op, p.base_step + t - 1, res[v]);
        if (!(qin && ((xin >> v) & 1))) {  // the Dirichlet ring stays zero
#pragma unroll
          for (int f = 0; f < NS; ++f) res[v][f] = 0.0f;
        }
      }
      if (t < T) {
#pragma unroll
        for (int f = 0; f < NS; ++f)
#pragma unroll
          for (int v = 0; v < V; ++v) Rg[t < T ? t : 0][f][PH][v] = res[v][f];
      } else if (q >= ys && q < ye && wx) {
#pragma unroll
        for (int f = 0; f < NS; ++f) {
          float* dst = p.out[f] + (int64_t)q * sy + gx;
          if (xall) {
            *reinterpret_cast<float4*>(dst) = make_float4(res[0][f], res[1][f], res[2][f], res[3][f]);
          } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
              if ((xin >> v) & 1) dst[v] = res[v][f];
          }
        }
      }
    }
  };

  int r = 0;
  if constexpr (D == 3) {
    for (; r + 2 < nit; r += 3) {
      step(PhaseG<0>{}, r);
      step(PhaseG<1>{}, r + 1);
      step(PhaseG<2>{}, r + 2);
    }
    if (r < nit) step(PhaseG<0>{}, r++);
    if (r < nit) step(PhaseG<1>{}, r++);
  } else {
    static_assert(D == 5, "radius 1 or 2");
    for (; r + 4 < nit; r += 5) {
      step(PhaseG<0>{}, r);
      step(PhaseG<1>{}, r + 1);
      step(PhaseG<2>{}, r + 2);
      step(PhaseG<3>{}, r + 3);
      step(PhaseG<4>{}, r + 4);
    }
    if (r < nit) step(PhaseG<0>{}, r++);
    if (r < nit) step(PhaseG<1>{}, r++);
    if (r < nit) step(PhaseG<2>{}, r++);
    if (r < nit) step(PhaseG<3>{}, r++);
  }
}

// ------------------------------------------------------------------------
// FDTD-2D, y-streamed in its two phases.  The fused update (OpFdtd2D::apply)
// evaluates E' four times per cell -- at the cell, Ex' at x+1 and Ey' at y+1
// -- because it sees only the previous level.  Streaming along y, level t can
// instead compute E' of row q+1 (one row ahead) once per cell and keep it for
// the next iteration, where it is that level's own E' of row q: H' of row q
// then takes Ex'(q) at x and x+1 and Ey' at q and q+1 from registers.  Every
// E' and H' value is the same expression on the same operands as in the fused
// form (bit-identical results); per cell and level it is two E' evaluations
// instead of four, and two shuffles instead of eighteen.
//
// Per level t >= 1 and iteration (row k = kb + r):
//   E'(qE = k - t + 1) from level t-1's row qE (Ex, Ey, Hz) and Hz(qE - 1);
//   H'(qH = k - t)     from level t-1's Hz(qH), this level's E'(qH) (computed
//                      one iteration earlier) and Ey'(qE);
//   level t's output row qH = (Ex'(qH), Ey'(qH), H'(qH)).
// Registers alternate between two slots with the iteration parity (PH), so
// no row is ever copied.
template <int T>
__global__ void __launch_bounds__(kStream2dThreads)
    stream2d_fdtd_kernel(const __grid_constant__ Stream2dgParams p) {
  constexpr int V = 4, HX = (T + 3) / 4 * 4;
  constexpr int RPBX = kStream2dWidth - 2 * HX;
  static_assert(RPBX >= 4, "depth");
  grid_dependency_sync();
  const int w = blockIdx.x * (kStream2dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.ntx * p.nseg) return;  // whole warps only
  const int strip = w % p.ntx, seg = w / p.ntx;
  const int lane = threadIdx.x & 31;
  const int nx = p.L.n0, ny = p.L.n1;
  const int64_t sy = p.L.sy;
  const int gx = strip * RPBX - HX + V * lane;  // multiple of 4
  unsigned xin = 0;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if ((unsigned)(gx + v) < (unsigned)nx) xin |= 1u << v;
  const bool xall = xin == 0xFu;
  const bool wx = V * lane >= HX && V * lane < HX + RPBX;
  const int ys = seg * p.zseg;
  const int ye = min(ny, ys + p.zseg);
  const int kb = ys - T;
  const int nit = (ye + T - 1) - kb + 1;
  const bool src_row = p.op.variant == 0;  // Ey on interior row 0 driven to the step index

  auto load4 = [&](const float* base, int k, float (&d)[V]) {
#pragma unroll
    for (int v = 0; v < V; ++v) d[v] = 0.0f;
    if ((unsigned)k < (unsigned)ny) {
      const float* src = base + (int64_t)k * sy + gx;
      if (xall) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(src));
        d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if ((xin >> v) & 1) d[v] = __ldg(src + v);
      }
    }
  };

  float In[2][3][V];       // level 0: input rows k (slot PH) and k - 1 (slot PH ^ 1)
  float Pf[2][3][V];       // input rows fetched ahead (k + 1 in slot PH ^ 1, k + 2 in PH)
  float Ec[T + 1][2][2][V];  // level t: E' rows (slot PH: row k - t + 1; PH ^ 1: row k - t)
  float Hl[T + 1][2][V];     // level t: H' rows (slot PH: row k - t; PH ^ 1: row k - t - 1)
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int v = 0; v < V; ++v) {
#pragma unroll
      for (int f = 0; f < 3; ++f) In[s][f][v] = 0.0f;
#pragma unroll
      for (int t = 0; t <= T; ++t) {
        Ec[t][s][0][v] = Ec[t][s][1][v] = 0.0f;
        Hl[t][s][v] = 0.0f;
      }
    }
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int f = 0; f < 3; ++f) load4(p.in[f], kb + j, Pf[j][f]);

  // EDG: some level's row of this iteration may lie outside [0, ny) and is
  // zeroed; otherwise every level's rows are inside and only x is tested
  auto step = [&](auto ph, auto edg, int r) {
    constexpr int PH = decltype(ph)::value, PO = PH ^ 1;
    constexpr bool EDG = decltype(edg)::value != 0;
    const int k = kb + r;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
#pragma unroll
      for (int v = 0; v < V; ++v) In[PH][f][v] = Pf[PH][f][v];
      load4(p.in[f], k + 2, Pf[PH][f]);
    }
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int qE = k - t + 1, qH = k - t;
      // level t-1's row qE (Ex, Ey, Hz) and its Hz of row qE - 1 = qH
      const float(&Lx)[V] = t == 1 ? In[PH][0] : Ec[t > 1 ? t - 1 : 0][PO][0];
      const float(&Ly)[V] = t == 1 ? In[PH][1] : Ec[t > 1 ? t - 1 : 0][PO][1];
      const float(&Lh)[V] = t == 1 ? In[PH][2] : Hl[t > 1 ? t - 1 : 0][PH];
      const float(&Lhp)[V] = t == 1 ? In[PO][2] : Hl[t > 1 ? t - 1 : 0][PO];
      const int step_t = p.base_step + t - 1;
      // E' of row qE (OpFdtd2D::ex_new / ey_new at that row)
      const float hl = __shfl_up_sync(0xffffffffu, Lh[V - 1], 1);  // Hz(qE) at x - 1 of cell 0
      const bool qEin = !EDG || (unsigned)qE < (unsigned)ny;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const bool in = qEin && ((xin >> v) & 1);
        const float hxm = v > 0 ? Lh[v - 1] : hl;
        Ec[t][PH][0][v] = in ? Lx[v] - 0.5f * (Lh[v] - hxm) : 0.0f;
        Ec[t][PH][1][v] = !in ? 0.0f
                              : (src_row && qE == 0) ? (float)step_t
                                                     : Ly[v] - 0.5f * (Lh[v] - Lhp[v]);
      }
      // H' of row qH from E'(qH) (slot PO) and Ey'(qE)
      const float exr = __shfl_down_sync(0xffffffffu, Ec[t][PO][0][0], 1);  // Ex'(qH) at x + 1 of cell 3
      const bool qHin = !EDG || (unsigned)qH < (unsigned)ny;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const float ex = Ec[t][PO][0][v], ey = Ec[t][PO][1][v];
        const float exp1 = v < V - 1 ? Ec[t][PO][0][v + 1] : exr;
        float d = (exp1 - ex) + Ec[t][PH][1][v];
        d = (p.op.variant == 1) ? d + ey : d - ey;
        const float h = Lhp[v] - 0.7f * d;
        Hl[t][PH][v] = (qHin && ((xin >> v) & 1)) ? h : 0.0f;
      }
      if (t == T && qH >= ys && qH < ye && wx) {
        float* dst[3] = {p.out[0] + (int64_t)qH * sy + gx, p.out[1] + (int64_t)qH * sy + gx,
                         p.out[2] + (int64_t)qH * sy + gx};
        const float(&ox)[V] = Ec[T][PO][0];
        const float(&oy)[V] = Ec[T][PO][1];
        const float(&oh)[V] = Hl[T][PH];
        if (xall) {
          *reinterpret_cast<float4*>(dst[0]) = make_float4(ox[0], ox[1], ox[2], ox[3]);
          *reinterpret_cast<float4*>(dst[1]) = make_float4(oy[0], oy[1], oy[2], oy[3]);
          *reinterpret_cast<float4*>(dst[2]) = make_float4(oh[0], oh[1], oh[2], oh[3]);
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if ((xin >> v) & 1) {
              dst[0][v] = ox[v];
              dst[1][v] = oy[v];
              dst[2][v] = oh[v];
            }
        }
      }
    }
  };

  int r = 0;
  for (; r + 1 < nit; r += 2) {
    // the two iterations' level rows span [kb + r - T, kb + r + 1]
    if (kb + r - T >= 0 && kb + r + 1 < ny) {
      step(PhaseG<0>{}, PhaseG<0>{}, r);
      step(PhaseG<1>{}, PhaseG<0>{}, r + 1);
    } else {
      step(PhaseG<0>{}, PhaseG<1>{}, r);
      step(PhaseG<1>{}, PhaseG<1>{}, r + 1);
    }
  }
  if (r < nit) step(PhaseG<0>{}, PhaseG<1>{}, r);
}

// Rician-denoise-2D streamed in its two phases.  The fused update
// (OpRician2D::apply) recomputes g = 1/sqrt(eps + |grad u|^2) at the four
// neighbours of every cell, four rsqrt and ~200 more instructions per update;
// here every level computes g once per cell, one row ahead of its update, the
// order of the reference kernel (opencl/rician-denoise-2d/rician-denoise-2d.cpp:
// 271-275 then :292-329) and of the two-phase tile step.  The operations and
// their operands are those of OpRician2D::g_at and ::apply2, so the result is
// bit for bit the fused kernels'.
//
// Level t works on row q = k - 2t (the update reaches two rows: g of the rows
// beside q needs u two rows away).  At iteration k it first computes
// g_{t-1}(q + 1) from u_{t-1} rows q .. q + 2 -- row q + 2 is what level t-1
// produced this iteration -- then updates row q from u_{t-1} rows q - 1 .. q + 1,
// g_{t-1} rows q - 1 .. q + 1 and F(q).  Each level keeps the four newest rows
// of its u and of the g computed from them in registers, in slots that rotate
// with the iteration index (4 phases), so no row is copied.  Level t's F row
// for the next iteration is fetched as soon as this iteration's is used.
// FAST selects the division (ots_div): a template argument, so the kernel of
// one variant carries no code of the other.
template <int N>
struct PhaseR {
  static constexpr int value = N;
};

template <int T, bool FAST>
__global__ void __launch_bounds__(kStream2dThreads)
    stream2d_rician_kernel(const __grid_constant__ Stream2dgParams p) {
  constexpr int V = 4, R = 2, HX = (R * T + 3) / 4 * 4;
  constexpr int RPBX = kStream2dWidth - 2 * HX;
  static_assert(RPBX >= 4, "depth");
  constexpr float DT = 5.0f, SIGMA2 = 0.0025f, GAMMA = 0.065f / 0.0025f;
  grid_dependency_sync();
  const int w = blockIdx.x * (kStream2dThreads / 32) + (threadIdx.x >> 5);
  if (w >= p.ntx * p.nseg) return;  // whole warps only
  const int strip = w % p.ntx, seg = w / p.ntx;
  const int lane = threadIdx.x & 31;
  const int nx = p.L.n0, ny = p.L.n1;
  const int64_t sy = p.L.sy;
  const int gx = strip * RPBX - HX + V * lane;  // multiple of 4
  unsigned xin = 0;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if ((unsigned)(gx + v) < (unsigned)nx) xin |= 1u << v;
  const bool xall = xin == 0xFu;
  const bool wx = V * lane >= HX && V * lane < HX + RPBX;
  const int ys = seg * p.zseg;
  const int ye = min(ny, ys + p.zseg);
  const int kb = ys - R * T;
  const int nit = (ye + R * T - 1) - kb + 1;
  constexpr bool fast = FAST;
  const float* const F = p.aux[0];

  auto load4 = [&](const float* base, int k, float (&d)[V]) {
#pragma unroll
    for (int v = 0; v < V; ++v) d[v] = 0.0f;
    if ((unsigned)k < (unsigned)ny) {
      const float* src = base + (int64_t)k * sy + gx;
      if (xall) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(src));
        d[0] = a.x; d[1] = a.y; d[2] = a.z; d[3] = a.w;
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if ((xin >> v) & 1) d[v] = __ldg(src + v);
      }
    }
  };

  // U[t][s]: level t's rows (t = 0: the input), newest in slot (iteration % 4)
  // G[t][s]: g of level t's rows, g(row) in the slot of the iteration that
  // computed it (one iteration after the row itself)
  float U[T][4][V], G[T][4][V];
  float Pf[2][V];  // input rows fetched ahead
  float Ff[T][V];  // level t + 1's F row of the coming iteration
#pragma unroll
  for (int t = 0; t < T; ++t)
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int v = 0; v < V; ++v) U[t][s][v] = G[t][s][v] = 0.0f;
  load4(p.in[0], kb, Pf[0]);
  load4(p.in[0], kb + 1, Pf[1]);
#pragma unroll
  for (int t = 1; t <= T; ++t) load4(F, kb - R * t, Ff[t - 1]);

  auto step = [&](auto ph, int r) {
    constexpr int PH = decltype(ph)::value;
    constexpr int S0 = PH, S1 = (PH + 3) & 3, S2 = (PH + 2) & 3, S3 = (PH + 1) & 3;  // age 0..3
    const int k = kb + r;
#pragma unroll
    for (int v = 0; v < V; ++v) U[0][S0][v] = Pf[PH & 1][v];
    load4(p.in[0], k + 2, Pf[PH & 1]);
#pragma unroll
    for (int t = 1; t <= T; ++t) {
      const int q = k - R * t;
      // u_{t-1}: rows q+2 (age 0), q+1 (1), q (2), q-1 (3)
      const float(&up2)[V] = U[t - 1][S0];
      const float(&up1)[V] = U[t - 1][S1];
      const float(&u0)[V] = U[t - 1][S2];
      const float(&um1)[V] = U[t - 1][S3];
      // phase 1: g_{t-1}(q + 1) (OpRician2D::g_at at row q + 1)
      {
        const float l = __shfl_up_sync(0xffffffffu, up1[V - 1], 1);
        const float rr = __shfl_down_sync(0xffffffffu, up1[0], 1);
        const bool rin = (unsigned)(q + 1) < (unsigned)ny;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const float c = up1[v];
          const float xp = v < V - 1 ? up1[v + 1] : rr;
          const float xm = v > 0 ? up1[v - 1] : l;
          const float g = ots_rsqrt(1.0E-20f + sq(c - xp) + sq(c - xm) + sq(c - up2[v]) +
                                    sq(c - u0[v]));
          G[t - 1][S0][v] = (rin && ((xin >> v) & 1)) ? g : 0.0f;
        }
      }
      // g_{t-1}: rows q+1 (slot S0, just computed), q (S1), q-1 (S2)
      const float(&gb)[V] = G[t - 1][S0];
      const float(&gc)[V] = G[t - 1][S1];
      const float(&gtp)[V] = G[t - 1][S2];
      // phase 2: the update of row q (OpRician2D::apply2)
      const float(&fq)[V] = Ff[t - 1];
      const float ul = __shfl_up_sync(0xffffffffu, u0[V - 1], 1);
      const float ur = __shfl_down_sync(0xffffffffu, u0[0], 1);
      const float gl_ = __shfl_up_sync(0xffffffffu, gc[V - 1], 1);
      const float gr_ = __shfl_down_sync(0xffffffffu, gc[0], 1);
      const bool qin = (unsigned)q < (unsigned)ny;
      float o[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const float c = u0[v], f = fq[v];
        float rv = ots_div(c * f, SIGMA2, fast);
        rv = ots_div(rv * (2.38944f + rv * (0.950037f + rv)),
                     4.65314f + rv * (2.57541f + rv * (1.48937f + rv)), fast);
        const float gl = v > 0 ? gc[v - 1] : gl_;
        const float gr = v < V - 1 ? gc[v + 1] : gr_;
        const float gt = gtp[v], g_b = gb[v];
        const float ugl = (v > 0 ? u0[v - 1] : ul) * gl;
        const float ugr = (v < V - 1 ? u0[v + 1] : ur) * gr;
        const float ugt = um1[v] * gt, ugb = up1[v] * g_b;
        const float res = ots_div(c + DT * (ugb + ugt + ugr + ugl + GAMMA * f * rv),
                                  1.0f + DT * (gr + gl + g_b + gt + GAMMA), fast);
        o[v] = (qin && ((xin >> v) & 1)) ? res : 0.0f;
      }
      load4(F, q + 1, Ff[t - 1]);
      if (t < T) {
#pragma unroll
        for (int v = 0; v < V; ++v) U[t][S0][v] = o[v];
      } else if (q >= ys && q < ye && wx) {
        float* dst = p.out[0] + (int64_t)q * sy + gx;
        if (xall) {
          *reinterpret_cast<float4*>(dst) = make_float4(o[0], o[1], o[2], o[3]);
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v)
            if ((xin >> v) & 1) dst[v] = o[v];
        }
      }
    }
  };

  int r = 0;
  for (; r + 3 < nit; r += 4) {
    step(PhaseR<0>{}, r);
    step(PhaseR<1>{}, r + 1);
    step(PhaseR<2>{}, r + 2);
    step(PhaseR<3>{}, r + 3);
  }
  if (r < nit) step(PhaseR<0>{}, r++);
  if (r < nit) step(PhaseR<1>{}, r++);
  if (r < nit) step(PhaseR<2>{}, r++);
}

}  // namespace ots
