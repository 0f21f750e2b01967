// Seeded per-cell velocity noise for the flow-past-sphere start state.
//
// The start state is feq(rho=1, u_in + noise) with uniform noise in [-amp, +amp) on each
// velocity component.  The noise is a counter-based hash of (seed, grid level, cell,
// component), so the host oracle, the reference build and the CUDA fill kernel produce
// bit-identical velocities: the hash is integer-only and the float steps below are each
// one correctly rounded operation (the CUDA side uses explicit _rn intrinsics so the
// compiler cannot contract them into an FMA).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PSL_HD __host__ __device__ __forceinline__
#else
#define PSL_HD inline
#endif

// "lowbias32" integer finaliser (Chris Wellons' hash-prospector, public domain).
PSL_HD uint32_t psl_mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Uniform in [0, 1) with 24 random bits: exactly representable in float.
PSL_HD float psl_noise_unit(uint32_t seed, uint32_t level, uint32_t cell, uint32_t comp) {
  const uint32_t h = psl_mix32(seed ^ psl_mix32(cell * 4u + comp + psl_mix32(level + 0x9e3779b9u)));
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

// u_base + amp * (2r - 1), rounded once in the product and once in the sum.
PSL_HD float psl_noisy_velocity(float u_base, float amp, uint32_t seed, uint32_t level, uint32_t cell,
                                uint32_t comp) {
  const float r = psl_noise_unit(seed, level, cell, comp);
  const float t = r * 2.0f - 1.0f;  // exact: r has 24 bits, the result has at most 24
#if defined(__CUDA_ARCH__)
  return __fadd_rn(u_base, __fmul_rn(t, amp));
#else
  volatile float prod = t * amp;  // keep the two roundings separate on every host compiler
  return u_base + prod;
#endif
}
