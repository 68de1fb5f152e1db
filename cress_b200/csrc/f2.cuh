// Packed FP32x2 arithmetic for sm_100a stencils (internal).  F2 holds the
// values of two neighbouring grid points; every operator is one packed
// instruction (add/sub/mul.rn.f32x2, fma.rn.f32x2) that rounds each lane
// exactly as the scalar instruction would, so a formula written over F2
// gives each point the value the scalar formula gives it.  Scalars (per-
// level constants) broadcast to both lanes.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cress {

struct F2 {
  float2 v;
};

__device__ __forceinline__ F2 f2(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 f2(float a) { return F2{make_float2(a, a)}; }

__device__ __forceinline__ uint64_t f2_bits(float2 v) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 f2_from_bits(uint64_t r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  uint64_t r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a.v)), "l"(f2_bits(b.v)));
  return F2{f2_from_bits(r)};
}
__device__ __forceinline__ F2 operator*(float s, F2 b) { return f2(s) * b; }
__device__ __forceinline__ F2 operator*(F2 a, float s) { return a * f2(s); }
__device__ __forceinline__ F2 operator+(F2 a, float s) { return a + f2(s); }
__device__ __forceinline__ F2 operator+(float s, F2 b) { return f2(s) + b; }
__device__ __forceinline__ F2 operator-(F2 a, float s) { return a - f2(s); }
__device__ __forceinline__ F2 operator-(float s, F2 b) { return f2(s) - b; }
__device__ __forceinline__ F2 fmax2(F2 a, float s) { return f2(fmaxf(a.v.x, s), fmaxf(a.v.y, s)); }

// Per-point choice: the lanes whose bit is set in mask (bit 0 the first
// point, bit 1 the second) take a, the others b.  The float overload serves
// one-point code (bit 0).
__device__ __forceinline__ F2 sel2(int mask, F2 a, F2 b) {
  return f2((mask & 1) ? a.v.x : b.v.x, (mask & 2) ? a.v.y : b.v.y);
}
__device__ __forceinline__ float sel2(int mask, float a, float b) { return (mask & 1) ? a : b; }

// Two consecutive floats at an 8-byte aligned shared-memory address.
__device__ __forceinline__ F2 ld2(const float* p) { return F2{*reinterpret_cast<const float2*>(p)}; }

// The pair (p[dx], p[dx+1]) for a compile-time dx, from aligned pairs only
// (p itself 8-byte aligned): an odd dx combines the halves of the aligned
// pairs on either side.
__device__ __forceinline__ F2 pair_at(const float* p, int dx) {
  if ((dx & 1) == 0) return ld2(p + dx);
  const F2 a = ld2(p + dx - 1), b = ld2(p + dx + 1);
  return f2(a.v.y, b.v.x);
}

}  // namespace cress
