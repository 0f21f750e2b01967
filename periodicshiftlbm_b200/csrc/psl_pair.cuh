// A pair of FP32 lanes as one arithmetic value: every +, - and * is one packed sm_100
// instruction for both lanes (FADD2 / FMUL2 / FFMA2 through __fadd2_rn, __fmul2_rn,
// __ffma2_rn), each lane rounded exactly as the scalar FP32 operation rounds it.  The
// 16-bit update kernels collide two cells per thread in this type (psl_collision_g.cuh).
// F1 is the same arithmetic on one lane (explicitly rounded operations, which the compiler
// does not contract into FMAs), so a cell collided alone gives the bits of the same cell
// collided in a pair.
#pragma once
#include <cuda_runtime.h>

namespace psl {

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ explicit F2(float2 x) : v(x) {}
};

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a) { return F2(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))); }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }
// the operations of the templated collision (psl_collision_g.cuh) on pairs
__device__ __forceinline__ F2 gfma(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ F2 grecip(F2 a) { return F2(1.f / a.v.x, 1.f / a.v.y); }  // per lane
__device__ __forceinline__ F2 gsqrt(F2 a) { return F2(sqrtf(a.v.x), sqrtf(a.v.y)); }  // per lane
__device__ __forceinline__ bool all_zero(F2 a) { return a.v.x == 0.f && a.v.y == 0.f; }
__device__ __forceinline__ F2 sel_zero(F2 c, F2 if_zero, F2 other) {
  return F2(c.v.x == 0.f ? if_zero.v.x : other.v.x, c.v.y == 0.f ? if_zero.v.y : other.v.y);
}

struct F1 {
  float v;
  F1() = default;
  __device__ __forceinline__ F1(float s) : v(s) {}
};
__device__ __forceinline__ F1 operator+(F1 a, F1 b) { return F1(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ F1 operator-(F1 a) { return F1(-a.v); }
__device__ __forceinline__ F1 operator-(F1 a, F1 b) { return F1(__fadd_rn(a.v, -b.v)); }
__device__ __forceinline__ F1 operator*(F1 a, F1 b) { return F1(__fmul_rn(a.v, b.v)); }
__device__ __forceinline__ F1 gfma(F1 a, F1 b, F1 c) { return F1(__fmaf_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ F1 grecip(F1 a) { return F1(1.f / a.v); }
__device__ __forceinline__ F1 gsqrt(F1 a) { return F1(sqrtf(a.v)); }
__device__ __forceinline__ bool all_zero(F1 a) { return a.v == 0.f; }
__device__ __forceinline__ F1 sel_zero(F1 c, F1 if_zero, F1 other) { return c.v == 0.f ? if_zero : other; }

}  // namespace psl
