// Explicitly rounded arithmetic for code that must round exactly like the reference's
// host build: each call is one IEEE round-to-nearest operation, which the compiler may
// not fuse into an FMA (on the device the _rn intrinsics forbid contraction; on the host
// the oracle and reference builds use no FMA contraction).
#pragma once

#ifndef PSL_HDI
#if defined(__CUDACC__)
#define PSL_HDI __host__ __device__ __forceinline__
#else
#define PSL_HDI inline
#endif
#endif

namespace psl {

PSL_HDI float rn_add(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
PSL_HDI float rn_sub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
PSL_HDI float rn_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
PSL_HDI float rn_div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}
PSL_HDI double rn_add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
PSL_HDI double rn_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
PSL_HDI double rn_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
PSL_HDI double rn_div(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}

}  // namespace psl
