// Pairs of nodes in one instruction: sm_100's packed f32x2 add, subtract, multiply and
// fused multiply-add, written as PTX. Each lane rounds as the scalar operation does
// (IEEE round to nearest, subnormals kept), so arithmetic on pairs is bit for bit the
// scalar arithmetic -- with one caution, measured on sm_100a: ptxas contracts a packed
// product into the packed sum it feeds (one rounding where the source has two), whatever
// --fmad says. A product that a sum consumes is therefore formed lane by lane by its
// caller; a product that is an FMA's addend cannot be contracted and stays packed.
#pragma once

#include <cuda_runtime.h>

namespace cwb {

__device__ __forceinline__ unsigned long long f2_bits(const float2 v) {
  return *reinterpret_cast<const unsigned long long *>(&v);
}
__device__ __forceinline__ float2 f2_of(const unsigned long long v) {
  return *reinterpret_cast<const float2 *>(&v);
}
__device__ __forceinline__ float2 p_add(const float2 a, const float2 b) {
  unsigned long long r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_of(r);
}
__device__ __forceinline__ float2 p_sub(const float2 a, const float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_of(r);
}
__device__ __forceinline__ float2 p_mul(const float2 a, const float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_of(r);
}
__device__ __forceinline__ float2 p_fma(const float2 a, const float2 b, const float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return f2_of(r);
}
__device__ __forceinline__ float2 p_splat(const float v) { return make_float2(v, v); }

// D+ of a pair: u(1) - uc, times w0 (R > 1), then w_{k-1} (u(k) - u(1-k)) fused in for
// k = 2 .. R (dplus in step.cuh, lane by lane)
template <int R, class Tap>
__device__ __forceinline__ float2 p_dplus(const Tap &u, const float2 uc, const float2 *w) {
  float2 d = p_sub(u(1), uc);
  if (R > 1)
    d = p_mul(w[0], d);
#pragma unroll
  for (int k = 2; k <= R; ++k)
    d = p_fma(w[k - 1], p_sub(u(k), u(1 - k)), d);
  return d;
}

}  // namespace cwb
