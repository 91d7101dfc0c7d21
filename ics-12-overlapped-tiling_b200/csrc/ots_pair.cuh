// ots_pair.cuh -- packed FP32 pairs in 64-bit registers (sm_100 f32x2
// instructions: two IEEE round-to-nearest operations in one instruction, bit
// for bit the scalar results), shared by the packed 3D and 2D stream kernels.
#pragma once

#include <stdint.h>

namespace ots {

__device__ __forceinline__ uint64_t p2_make(float lo, float hi) {
  uint64_t d;
  asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
  return d;
}
__device__ __forceinline__ float p2_lo(uint64_t a) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a));
  (void)hi;
  return lo;
}
__device__ __forceinline__ float p2_hi(uint64_t a) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a));
  (void)lo;
  return hi;
}
__device__ __forceinline__ uint64_t p2_add(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t p2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
// both halves of a pair ANDed with one 32-bit mask (two 32-bit ANDs: no
// 64-bit mask pair has to be assembled)
__device__ __forceinline__ uint64_t p2_and(uint64_t a, uint32_t m) {
  uint64_t d;
  asm("{.reg .b32 l, h; mov.b64 {l, h}, %1; and.b32 l, l, %2; and.b32 h, h, %2;"
      " mov.b64 %0, {l, h};}"
      : "=l"(d)
      : "l"(a), "r"(m));
  return d;
}
// the low half ANDed with mlo, the high half with mhi
__device__ __forceinline__ uint64_t p2_and2(uint64_t a, uint32_t mlo, uint32_t mhi) {
  uint64_t d;
  asm("{.reg .b32 l, h; mov.b64 {l, h}, %1; and.b32 l, l, %2; and.b32 h, h, %3;"
      " mov.b64 %0, {l, h};}"
      : "=l"(d)
      : "l"(a), "r"(mlo), "r"(mhi));
  return d;
}
// 16 bytes of shared memory as two pairs, and back
__device__ __forceinline__ void p2_lds(const float* a, uint64_t& x, uint64_t& y) {
  const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(a);
  x = v.x;
  y = v.y;
}
// two 8-byte stores: each pair is already an aligned register pair, so no
// move is needed to assemble a 16-byte (4-register) source
__device__ __forceinline__ void p2_sts(float* a, uint64_t x, uint64_t y) {
  reinterpret_cast<uint64_t*>(a)[0] = x;
  reinterpret_cast<uint64_t*>(a)[1] = y;
}
// 16 bytes of shared memory in natural order (v0, v1, v2, v3) as the pairs
// (v0, v2) and (v1, v3)
__device__ __forceinline__ void p2_lds_nat(const float* a, uint64_t& x, uint64_t& y) {
  const float4 v = *reinterpret_cast<const float4*>(a);
  x = p2_make(v.x, v.z);
  y = p2_make(v.y, v.w);
}

}  // namespace ots
