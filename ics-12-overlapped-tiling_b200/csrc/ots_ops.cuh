// ots_ops.cuh -- per-point updates of the thirteen stencils.
//
// Every stencil is written as ONE fused update of its evolving fields from
// the previous time level, so that every kernel family (overlapped tile,
// z-streamed tile, plain one-step) shares the same arithmetic.  Multi-phase
// reference kernels are fused by recomputing the first phase at the
// neighbours the second phase reads: fdtd-2d recomputes E' at x+1 and y+1
// (opencl/fdtd-2d/fdtd-2d.cpp:267-330), rician-denoise-2d recomputes g at the
// four neighbours (opencl/rician-denoise-2d/rician-denoise-2d.cpp:271-329).
// Recomputation repeats the identical operations, so the fused result is bit
// for bit the phased one.  The overlapped tile runs Rician in its two phases
// (TWO_PHASE: g once per tile cell in shared memory), which measured 17 %
// faster; TV's shared rsqrt terms did not pay for the extra barrier.
//
// Operand order follows the reference exactly (the CPU loops where they are
// correct, else the generated kernels).  The library is compiled with
// -fmad=false, so every + and * is its own IEEE single operation and linear
// stencils reproduce the CPU result exactly.  1/sqrt terms use rsqrtf as the
// reference kernels used OpenCL rsqrt.
//
// Accessor contract (A):   a(f, dz, dy, dx)      state field f at an offset
//                          a.inside(dz, dy, dx)  is that cell in the domain
// Cells outside the domain hold 0 for every field (zero Dirichlet ring).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#if defined(__CUDACC__)
#define OTS_HD __host__ __device__ __forceinline__
#else
#define OTS_HD inline
#endif

namespace ots {

// 1/sqrt: the approximate rsqrt on the GPU (as the reference kernels used
// OpenCL rsqrt); on the host (the runner's own -v check) 1/sqrtf.  Every
// argument here is eps + a sum of squares with eps >= 1e-20, a normal float,
// and the result is at most 1e10, also normal; on that range the
// flush-to-zero form of the instruction returns exactly what rsqrtf returns
// (compared on B200 for all 1.63e9 floats in [1e-20, +inf): no difference)
// without rsqrtf's handling of subnormal arguments.
OTS_HD float ots_rsqrt(float v) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
#else
  return 1.0f / sqrtf(v);
#endif
}

struct OpArgs {
  float coef;   // averaging weight
  float h2;     // Poisson h^2
  int variant;  // 0 baseline, 1 reference arithmetic, 2 fast division
};

// Division: IEEE, or in the fast variant the approximate PTX division
// (div.approx.ftz.f32: maximum error 2 ulp for |b| in [2^-126, 2^126],
// subnormal operands and results flushed to zero); the host (the runner's
// own -v check) divides exactly.
OTS_HD float ots_div(float a, float b, bool fast) {
#if defined(__CUDA_ARCH__)
  if (fast) {
    float q;
    asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(q) : "f"(a), "f"(b));
    return q;
  }
  return a / b;
#else
  (void)fast;
  return a / b;
#endif
}

OTS_HD float sq(float v) { return v * v; }

#if defined(__CUDACC__)
// Packed FP32 (sm_100 add/sub/mul .f32x2): two IEEE round-to-nearest
// operations per instruction, so results equal the scalar ones bit for bit.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 p, q, d; mov.b64 p, {%2,%3}; mov.b64 q, {%4,%5}; add.rn.f32x2 d, p, q;"
      " mov.b64 {%0,%1}, d;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 p, q, d; mov.b64 p, {%2,%3}; mov.b64 q, {%4,%5}; sub.rn.f32x2 d, p, q;"
      " mov.b64 {%0,%1}, d;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 r;
  asm("{.reg .b64 p, q, d; mov.b64 p, {%2,%3}; mov.b64 q, {%4,%5}; mul.rn.f32x2 d, p, q;"
      " mov.b64 {%0,%1}, d;}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
#endif

// ---------------------------------------------------------------- 1D ----

// opencl/jacobi-1d/jacobi-1d.cpp:635-637
struct OpJacobi1D {
  static constexpr int DIMS = 1, NS = 1, NA = 0, RX = 1, RY = 0, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    o[0] = p.coef * (a(0, 0, 0, -1) + a(0, 0, 0, 0) + a(0, 0, 0, 1));
  }
};

// opencl/jacobi-1d-5pt/jacobi-1d-5pt.cpp:507-511 (CPU arithmetic; the
// generated kernel's step 1 is defective, jacobi-1d-5pt.cpp:197-206)
struct OpJacobi1D5 {
  static constexpr int DIMS = 1, NS = 1, NA = 0, RX = 2, RY = 0, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    o[0] = p.coef *
           (a(0, 0, 0, -2) + a(0, 0, 0, -1) + a(0, 0, 0, 0) + a(0, 0, 0, 1) + a(0, 0, 0, 2));
  }
};

// opencl/jacobi-1d-7pt/jacobi-1d-7pt.cpp:515-521 (weight 0.2f as written)
struct OpJacobi1D7 {
  static constexpr int DIMS = 1, NS = 1, NA = 0, RX = 3, RY = 0, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    o[0] = p.coef * (a(0, 0, 0, -3) + a(0, 0, 0, -2) + a(0, 0, 0, -1) + a(0, 0, 0, 0) +
                     a(0, 0, 0, 1) + a(0, 0, 0, 2) + a(0, 0, 0, 3));
  }
};

// ---------------------------------------------------------------- 2D ----

// opencl/jacobi-2d/jacobi-2d.cpp:824-828: (1/5)(l + c + r + t + b)
struct OpJacobi2D {
  static constexpr int DIMS = 2, NS = 1, NA = 0, RX = 1, RY = 1, RZ = 0;
  static constexpr bool STAR = true;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    o[0] = p.coef *
           (a(0, 0, 0, -1) + a(0, 0, 0, 0) + a(0, 0, 0, 1) + a(0, 0, -1, 0) + a(0, 0, 1, 0));
  }
  // Same arithmetic from the five values (used by the y-streamed kernel).
  OTS_HD static float star2d(float xm, float c, float xp, float ym, float yp, float,
                             const OpArgs& p) {
    return p.coef * (xm + c + xp + ym + yp);
  }
};

// Reference: opencl/poisson-2d/poisson-2d.cpp:644-648, 8c - (8 neighbours).
// Baseline: Jacobi sweep for the 5-point Poisson problem, (sum4 - h^2 f)/4.
struct OpPoisson2D {
  static constexpr int DIMS = 2, NS = 1, NA = 1, RX = 1, RY = 1, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static void apply(const A& a, const float* aux, const OpArgs& p,
                                               int, float* o) {
    if (p.variant == 1) {
      o[0] = 8.0f * a(0, 0, 0, 0) -
             (a(0, 0, -1, -1) + a(0, 0, -1, 0) + a(0, 0, -1, 1) + a(0, 0, 0, -1) +
              a(0, 0, 0, 1) + a(0, 0, 1, -1) + a(0, 0, 1, 0) + a(0, 0, 1, 1));
    } else {
      float s = a(0, 0, -1, 0) + a(0, 0, 0, -1) + a(0, 0, 0, 1) + a(0, 0, 1, 0);
      o[0] = (s - p.h2 * aux[0]) * 0.25f;
    }
  }
  // Baseline variant only (the reference variant is 9-point).
  OTS_HD static float star2d(float xm, float, float xp, float ym, float yp, float f,
                             const OpArgs& p) {
    float s = ym + xm + xp + yp;
    return (s - p.h2 * f) * 0.25f;
  }
};

// opencl/gradient-2d/gradient-2d.cpp:283-289: c + rsqrt(1e-4 + sum (c-n)^2)
struct OpGradient2D {
  static constexpr int DIMS = 2, NS = 1, NA = 0, RX = 1, RY = 1, RZ = 0;
  static constexpr bool STAR = true;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs&, int,
                                               float* o) {
    float c = a(0, 0, 0, 0);
    o[0] = c + ots_rsqrt(0.0001f + sq(c - a(0, 0, 0, -1)) + sq(c - a(0, 0, 0, 1)) +
                      sq(c - a(0, 0, -1, 0)) + sq(c - a(0, 0, 1, 0)));
  }
  OTS_HD static float star2d(float xm, float c, float xp, float ym, float yp, float,
                             const OpArgs&) {
    return c + ots_rsqrt(0.0001f + sq(c - xm) + sq(c - xp) + sq(c - ym) + sq(c - yp));
  }
};

// Fields: 0 Ex, 1 Ey, 2 Hz.  opencl/fdtd-2d/fdtd-2d.cpp:267-330.
// Baseline: standard sign (Hz -= 0.7(dEx/dx + dEy/dy)) and Ey on interior row
// 0 driven to the global step index.  Reference: "+Ey" (fdtd-2d.cpp:322), no
// source.
struct OpFdtd2D {
  static constexpr int DIMS = 2, NS = 3, NA = 0, RX = 1, RY = 1, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static float ey_new(const A& a, const OpArgs& p, int t, int dy,
                                                 int dx) {
    if (!a.inside(0, dy, dx)) return 0.0f;
    if (p.variant == 0 && a.gy() + dy == 0) return (float)t;
    return a(1, 0, dy, dx) - 0.5f * (a(2, 0, dy, dx) - a(2, 0, dy - 1, dx));
  }
  template <class A>
  OTS_HD static float ex_new(const A& a, int dy, int dx) {
    if (!a.inside(0, dy, dx)) return 0.0f;
    return a(0, 0, dy, dx) - 0.5f * (a(2, 0, dy, dx) - a(2, 0, dy, dx - 1));
  }
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int t,
                                               float* o) {
    float ey = ey_new(a, p, t, 0, 0);
    float ex = ex_new(a, 0, 0);
    float exr = ex_new(a, 0, 1);
    float eyb = ey_new(a, p, t, 1, 0);
    float d = (exr - ex) + eyb;
    d = (p.variant == 1) ? d + ey : d - ey;
    o[0] = ex;
    o[1] = ey;
    o[2] = a(2, 0, 0, 0) - 0.7f * d;
  }
};

// opencl/rician-denoise-2d/rician-denoise-2d.cpp:153-161 constants, :271-329
// arithmetic; aux 0 = F (the noisy image).
struct OpRician2D {
  static constexpr int DIMS = 2, NS = 1, NA = 1, RX = 2, RY = 2, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static float g_at(const A& a, int dy, int dx) {
    if (!a.inside(0, dy, dx)) return 0.0f;
    float c = a(0, 0, dy, dx);
    return ots_rsqrt(1.0E-20f + sq(c - a(0, 0, dy, dx + 1)) + sq(c - a(0, 0, dy, dx - 1)) +
                  sq(c - a(0, 0, dy + 1, dx)) + sq(c - a(0, 0, dy - 1, dx)));
  }
  template <class A>
  OTS_HD static void apply(const A& a, const float* aux, const OpArgs& p, int,
                                               float* o) {
    const float DT = 5.0f, SIGMA2 = 0.0025f, GAMMA = 0.065f / 0.0025f;
    const bool fast = p.variant == 2;
    float c = a(0, 0, 0, 0), f = aux[0];
    float r = ots_div(c * f, SIGMA2, fast);
    r = ots_div(r * (2.38944f + r * (0.950037f + r)),
                4.65314f + r * (2.57541f + r * (1.48937f + r)), fast);
    float gl = g_at(a, 0, -1), gr = g_at(a, 0, 1), gt = g_at(a, -1, 0), gb = g_at(a, 1, 0);
    float ugl = a(0, 0, 0, -1) * gl, ugr = a(0, 0, 0, 1) * gr, ugt = a(0, 0, -1, 0) * gt,
          ugb = a(0, 0, 1, 0) * gb;
    o[0] = ots_div(c + DT * (ugb + ugt + ugr + ugl + GAMMA * f * r),
                   1.0f + DT * (gr + gl + gb + gt + GAMMA), fast);
  }
  // Two-phase form for the overlapped tile, the reference kernel's own order
  // (:271-275 then :292-329): phase 1 stores g once per tile cell, phase 2
  // reads it at the four neighbours -- the same values g_at recomputes.
  static constexpr bool TWO_PHASE = true;
  static constexpr int G_LO = 1, G_HI = 1;  // g on the tile minus its outer ring
  template <class A>
  OTS_HD static float phase1(const A& a) { return g_at(a, 0, 0); }
  template <class A, class G>
  OTS_HD static void apply2(const A& a, const G& g, const float* aux, const OpArgs& p, int,
                            float* o) {
    const float DT = 5.0f, SIGMA2 = 0.0025f, GAMMA = 0.065f / 0.0025f;
    const bool fast = p.variant == 2;
    float c = a(0, 0, 0, 0), f = aux[0];
    float r = ots_div(c * f, SIGMA2, fast);
    r = ots_div(r * (2.38944f + r * (0.950037f + r)),
                4.65314f + r * (2.57541f + r * (1.48937f + r)), fast);
    float gl = g(0, -1), gr = g(0, 1), gt = g(-1, 0), gb = g(1, 0);
    float ugl = a(0, 0, 0, -1) * gl, ugr = a(0, 0, 0, 1) * gr, ugt = a(0, 0, -1, 0) * gt,
          ugb = a(0, 0, 1, 0) * gb;
    o[0] = ots_div(c + DT * (ugb + ugt + ugr + ugl + GAMMA * f * r),
                   1.0f + DT * (gr + gl + gb + gt + GAMMA), fast);
  }
};

// opencl/cdsc-tv-update-2d/cdsc-tv-update-2d.cpp:163-164, :287-309;
// aux 0 = F, aux 1 = V.
struct OpTvUpdate2D {
  static constexpr int DIMS = 2, NS = 1, NA = 2, RX = 1, RY = 1, RZ = 0;
  static constexpr bool STAR = false;
  template <class A>
  OTS_HD static void apply(const A& a, const float* aux, const OpArgs& p, int,
                                               float* o) {
    const float EPI1 = 1e-8f, ALPHA = 1.1f;
    const bool fast = p.variant == 2;
    float tc = a(0, 0, -1, 0), tr = a(0, 0, -1, 1), ml = a(0, 0, 0, -1), mc = a(0, 0, 0, 0),
          mr = a(0, 0, 0, 1), bl = a(0, 0, 1, -1), bc = a(0, 0, 1, 0);
    float F = aux[0], V = aux[1];
    float c1 =
        ots_div(mc * ots_rsqrt(EPI1 + ((bc - mc) * (bc - mc)) + ((mr - mc) * (mr - mc))), V, fast);
    float c2 =
        ots_div(mc * ots_rsqrt(EPI1 + ((mc - tc) * (mc - tc)) + ((tr - tc) * (tr - tc))), V, fast);
    float c3 =
        ots_div(mc * ots_rsqrt(EPI1 + ((bc - mc) * (bc - mc)) + ((mr - mc) * (mr - mc))), V, fast);
    float c4 =
        ots_div(mc * ots_rsqrt(EPI1 + ((bl - ml) * (bl - ml)) + ((mc - ml) * (mc - ml))), V, fast);
    o[0] = ots_div(1.0f, ALPHA + c1 + c2 + c3 + c4, fast) *
           (ALPHA * F + c1 * bc + c2 * tc + c3 * mr + c4 * ml);
  }
};

// ---------------------------------------------------------------- 3D ----

// Generated-kernel operand order (opencl/jacobi-3d/jacobi-3d.cpp:282-304):
// x-1, c, x+1, y-1, y+1, z-1, z+1.
struct OpJacobi3D {
  static constexpr int DIMS = 3, NS = 1, NA = 0, RX = 1, RY = 1, RZ = 1;
  static constexpr bool STAR = true;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    o[0] = p.coef * (a(0, 0, 0, -1) + a(0, 0, 0, 0) + a(0, 0, 0, 1) + a(0, 0, -1, 0) +
                     a(0, 0, 1, 0) + a(0, -1, 0, 0) + a(0, 1, 0, 0));
  }
  // Same arithmetic from the seven values (used by the z-streamed kernels).
  OTS_HD static float star(float xm, float c, float xp, float ym, float yp,
                                               float zm, float zp, float, const OpArgs& p) {
    return p.coef * (xm + c + xp + ym + yp + zm + zp);
  }
  // Two neighbouring cells at once with packed FP32, same operation order.
  static constexpr bool PACKED = true;
#if defined(__CUDACC__)
  __device__ __forceinline__ static float2 star2(float2 xm, float2 c, float2 xp, float2 ym,
                                                 float2 yp, float2 zm, float2 zp, float2,
                                                 const OpArgs& p) {
    float2 s = add2(xm, c);
    s = add2(s, xp);
    s = add2(s, ym);
    s = add2(s, yp);
    s = add2(s, zm);
    s = add2(s, zp);
    return mul2(make_float2(p.coef, p.coef), s);
  }
#endif
};

// Reference: opencl/poisson-3d/poisson-3d.cpp:280-293, 26c - (26 neighbours,
// x outer, y, z inner).  Baseline: Jacobi sweep for the 7-point Poisson
// problem with RHS f: (x-1 + x+1 + y-1 + y+1 + z-1 + z+1 - h^2 f) * (1/6).
struct OpPoisson3D {
  static constexpr int DIMS = 3, NS = 1, NA = 1, RX = 1, RY = 1, RZ = 1;
  static constexpr bool STAR = true;  // star only in the baseline variant
  template <class A>
  OTS_HD static void apply(const A& a, const float* aux, const OpArgs& p,
                                               int, float* o) {
    if (p.variant == 1) {
      float s = 0.0f;
      bool first = true;
#pragma unroll
      for (int ox = -1; ox <= 1; ++ox)
#pragma unroll
        for (int oy = -1; oy <= 1; ++oy)
#pragma unroll
          for (int oz = -1; oz <= 1; ++oz) {
            if (ox == 0 && oy == 0 && oz == 0) continue;
            float v = a(0, oz, oy, ox);
            s = first ? v : s + v;
            first = false;
          }
      o[0] = 26.0f * a(0, 0, 0, 0) - s;
    } else {
      float s = a(0, 0, 0, -1) + a(0, 0, 0, 1) + a(0, 0, -1, 0) + a(0, 0, 1, 0) +
                a(0, -1, 0, 0) + a(0, 1, 0, 0);
      o[0] = (s - p.h2 * aux[0]) * (1.0f / 6.0f);
    }
  }
  OTS_HD static float star(float xm, float, float xp, float ym, float yp,
                                               float zm, float zp, float f, const OpArgs& p) {
    float s = xm + xp + ym + yp + zm + zp;
    return (s - p.h2 * f) * (1.0f / 6.0f);
  }
  // Scalar only: with packed FP32 the h^2 f product and the subtraction were
  // observed to round once (as a fused multiply-add) in rare cells.
  static constexpr bool PACKED = false;
#if defined(__CUDACC__)
  __device__ __forceinline__ static float2 star2(float2, float2, float2, float2, float2,
                                                 float2, float2, float2, const OpArgs&) {
    return make_float2(0.0f, 0.0f);
  }
#endif
};

// opencl/gradient-3d/gradient-3d.cpp:305-307
struct OpGradient3D {
  static constexpr int DIMS = 3, NS = 1, NA = 0, RX = 1, RY = 1, RZ = 1;
  static constexpr bool STAR = true;
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs&, int,
                                               float* o) {
    float c = a(0, 0, 0, 0);
    o[0] = c + ots_rsqrt(0.0001f + sq(c - a(0, 0, 0, -1)) + sq(c - a(0, 0, 0, 1)) +
                      sq(c - a(0, 0, -1, 0)) + sq(c - a(0, 0, 1, 0)) + sq(c - a(0, -1, 0, 0)) +
                      sq(c - a(0, 1, 0, 0)));
  }
  OTS_HD static float star(float xm, float c, float xp, float ym, float yp,
                                               float zm, float zp, float, const OpArgs&) {
    return c + ots_rsqrt(0.0001f + sq(c - xm) + sq(c - xp) + sq(c - ym) + sq(c - yp) +
                      sq(c - zm) + sq(c - zp));
  }
  static constexpr bool PACKED = false;  // 1/sqrt has no packed form
#if defined(__CUDACC__)
  __device__ __forceinline__ static float2 star2(float2, float2, float2, float2, float2, float2,
                                                 float2, float2, const OpArgs&) {
    return make_float2(0.0f, 0.0f);
  }
#endif
};

// opencl/cs-3d/cs-3d.cpp:161-163 constants, :284-308 arithmetic with y+1 as
// the "p1" direction throughout (the reference's step-1 code flips its two
// y-axis neighbours).  The generated text #defines eps as (1e-9), a double
// literal (:161), which makes each c term a double expression: the float
// squares are summed onto 1e-9 in double, 1/sqrt, multiplied by u and
// divided by 1.1f in double, and rounded to float once.  Double sqrt and
// division are IEEE on both the GPU and the host, so this stencil matches the
// CPU oracle bit for bit.
struct OpCs3D {
  static constexpr int DIMS = 3, NS = 1, NA = 0, RX = 1, RY = 1, RZ = 1;
  static constexpr bool STAR = false;
  OTS_HD static float cterm(float u, float a, float b, float c) {
    return (float)((double)u * (1.0 / sqrt(1e-9 + (double)a + (double)b + (double)c)) /
                   (double)1.1f);
  }
  // the fast variant: float 1/sqrt (rsqrt) and approximate division
  OTS_HD static float cterm_fast(float u, float a, float b, float c) {
    return ots_div(u * ots_rsqrt(1e-9f + a + b + c), 1.1f, true);
  }
  template <class A>
  OTS_HD static void apply(const A& a, const float*, const OpArgs& p, int,
                                               float* o) {
    const bool fast = p.variant == 2;
    const float ALPHA = 1.1f;
    float u = a(0, 0, 0, 0);
    float zp = a(0, 1, 0, 0), zm = a(0, -1, 0, 0), yp = a(0, 0, 1, 0), ym = a(0, 0, -1, 0),
          xp = a(0, 0, 0, 1), xm = a(0, 0, 0, -1);
    float zm_yp = a(0, -1, 1, 0), zm_xp = a(0, -1, 0, 1), zp_ym = a(0, 1, -1, 0),
          ym_xp = a(0, 0, -1, 1), zp_xm = a(0, 1, 0, -1), yp_xm = a(0, 0, 1, -1);
    float c1, c2, c3, c4;
    if (fast) {
      c1 = cterm_fast(u, sq(zp - u), sq(yp - u), sq(xp - u));
      c2 = cterm_fast(u, sq(u - zm), sq(zm_yp - zm), sq(zm_xp - zm));
      c3 = cterm_fast(u, sq(zp_ym - ym), sq(u - ym), sq(ym_xp - ym));
      c4 = cterm_fast(u, sq(zp_xm - xm), sq(yp_xm - xm), sq(u - xm));
    } else {
      c1 = cterm(u, sq(zp - u), sq(yp - u), sq(xp - u));
      c2 = cterm(u, sq(u - zm), sq(zm_yp - zm), sq(zm_xp - zm));
      c3 = cterm(u, sq(zp_ym - ym), sq(u - ym), sq(ym_xp - ym));
      c4 = cterm(u, sq(zp_xm - xm), sq(yp_xm - xm), sq(u - xm));
    }
    o[0] = ots_div(ALPHA * u + c1 * (zp + yp + xp) + c2 * zm + c3 * ym + c4 * xm,
                   ALPHA + 3.0f * c1 + c2 + c3 + c4, fast);
  }
};

}  // namespace ots
