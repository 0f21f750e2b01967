// The learned closure evaluated per warp inside the update kernel: 32 cells (one per
// lane) through the 10 -> 32 -> 32 -> 1 network with warp-level tensor-core MMAs
// (mma.sync m16n8k16, FP16 operands, FP32 accumulation).
//
// Why per warp inside the collision: the network sits between the two halves of a cell's
// collision (its input is the second-order moments, its output the relaxation rate), so
// every cell's whole collision state waits for it.  A CTA-wide tcgen05 MMA (psl_mlp.cuh)
// needs three CTA barriers and three MMA round trips per 128-cell tile, during which all
// of the CTA's warps wait; measured in the fused update kernel on the 256^3 turbulence box
// (FP16 storage) that ran at 10.7k MLUPS against 16.2k per warp and 25.6k with
// Smagorinsky.  Per warp there is no barrier: each warp's 28 MMAs complete in its own
// instruction stream while the SM's other warps keep their loads and arithmetic going.
// The CTA-wide tcgen05 path remains the closure's batched inference (psl_sgs_mlp_infer).
//
// Data flow per warp:
//   features -> normalised FP16 rows in shared memory, input 10 the constant 1 that
//   carries the layer-1 biases -> ldmatrix A fragments (2 M-tiles)
//   layer 1: 2 x 4 MMAs (K = 16); FP16 packing + ReLU (one cvt.rn.relu.f16x2 per pair)
//            turns the accumulators into the A fragments of layer 2 in registers (the
//            m16n8 accumulator layout of two adjacent N-tiles is the m16k16 A layout)
//   layer 2: 2 x 4 x 2 MMAs (K = 32), the biases entering as the first K-step's
//            accumulator input; packing + ReLU: the A fragments of layer 3
//   layer 3: 2 x 2 MMAs (N = 8, row 0 of W3 holds the output weights, b3 the input)
//   the output of row r sits in lane 4 (r % 8) (accumulator column 0); four shuffles bring
//   it to lane r, the lane that owns the cell.
// Weights stay in global memory (4.6 KB with the biases, L1-resident after the first warps), stored in
// fragment order: each lane reads its own B fragments of an N-tile pair with one 16-byte
// load, so no block copies them into shared memory and no block barrier waits for that copy.
// The normalisation, b3 and the output scale are kernel parameters (constant-bank operands).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "psl_mlp.cuh"

namespace psl {

constexpr int kXStride = 24;   // halves per feature row of a warp's tile (16 used)

// B fragments of mma.m16n8k16 (.col B = W^T, B[k][n] = W[n][k]): lane l = 4 g + t holds,
// for N-tile nt and K-step kk, b0 = (W[8nt+g][16kk+2t], W[8nt+g][16kk+2t+1]) and
// b1 = (W[8nt+g][16kk+8+2t], W[8nt+g][16kk+9+2t]), FP16 pairs, lower column in the low half.
struct MlpFrag {
  uint4 w1[2][32];     // [np][lane]: {b0, b1} of N-tile 2np, {b0, b1} of N-tile 2np+1; K = 16
                       // (inputs 0-9, input 10 the constant 1 times b1, 11-15 zero)
  uint4 w2[2][2][32];  // [kk][np][lane]
  uint4 w3[32];        // [lane]: {b0, b1} of K-step 0, {b0, b1} of K-step 1; row 0 = w3, rows 1-7 zero
  float4 b2[2][32];    // [kk][lane]: b2 at columns 16kk+2t, 16kk+2t+1, 16kk+8+2t, 16kk+9+2t
};

struct MlpScalars {
  float in_scale[kMlpIn];  // normalised feature = x * in_scale + in_offset
  float in_offset[kMlpIn];
  float b3;
  float out_scale;
};

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

// d += a b (accumulate) and d = a b (fresh accumulator: C is the zero register)
__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void mma16816_new(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                             uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%10,%10,%10};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1), "f"(0.f));
}

// d = a b + c with the accumulator input c given separately (the layer's biases)
__device__ __forceinline__ void mma16816_c(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                           uint32_t b0, uint32_t b1, float c0, float c1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%10,%11,%10,%11};"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1), "f"(c0), "f"(c1));
}

// (lo, hi) -> FP16 pair with ReLU, one instruction (cvt.rn.relu.f16x2.f32 puts its first
// source in the upper half); ReLU after rounding equals rounding after ReLU.
__device__ __forceinline__ uint32_t pack_relu(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}

// ReLU of the accumulators of N-tiles 2kk and 2kk+1 (columns 16kk..16kk+15) into the A
// fragment of K-step kk of the next layer.
__device__ __forceinline__ void acc_to_a(const float (&c0)[4], const float (&c1)[4], uint32_t (&a)[4]) {
  a[0] = pack_relu(c0[0], c0[1]);
  a[1] = pack_relu(c0[2], c0[3]);
  a[2] = pack_relu(c1[0], c1[1]);
  a[3] = pack_relu(c1[2], c1[3]);
}

// softplus(z) = ln(1 + e^z) from the fast exponential and logarithm: z itself above 15,
// e^z (1 - e^z / 2) below -7 (the next term of ln(1 + t) is t^3/3 < 3e-10 t there), and
// ln(1 + e^z) between, where the logarithm's absolute error (< 4e-7) is at most 4e-4 of
// the result.  nu_t moves by that fraction at most, tau = 3 (nu + nu_t) + 1/2 by 1e-7.
__device__ __forceinline__ float softplus_fast(float z) {
  const float t = __expf(z);
  return z > 15.f ? z : (z > -7.f ? __logf(1.f + t) : t * fmaf(-0.5f, t, 1.f));
}

// nu_t of this lane's cell.  All 32 lanes of the warp must call it (converged); `xtile`
// is the warp's 32 x kXStride FP16 staging tile in shared memory (16-byte aligned).
__device__ __forceinline__ float mlp_warp_eval(const MlpFrag* __restrict__ w, const MlpScalars& sc, __half* xtile,
                                               const float (&x)[kMlpIn]) {
  const int lane = threadIdx.x & 31;
  // normalised features -> FP16 row `lane` (K padded to 16 with zeros)
  {
    float xn[16];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) xn[i] = fmaf(x[i], sc.in_scale[i], sc.in_offset[i]);
    xn[kMlpIn] = 1.f;  // carries the layer-1 biases (W1 column 10)
#pragma unroll
    for (int i = kMlpIn + 1; i < 16; ++i) xn[i] = 0.f;
    uint32_t p[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const __half2 h = __floats2half2_rn(xn[2 * i], xn[2 * i + 1]);
      p[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    uint4* row = reinterpret_cast<uint4*>(xtile + lane * kXStride);
    row[0] = make_uint4(p[0], p[1], p[2], p[3]);
    row[1] = make_uint4(p[4], p[5], p[6], p[7]);
  }
  __syncwarp();
  const int m = lane >> 3, r = lane & 7;  // ldmatrix: this lane addresses row r of matrix m
  const uint32_t xs = mlp_smem_u32(xtile);
  const uint4 b3 = __ldg(&w->w3[lane]);  // W3's fragments for both K-steps
  const float4 bias0 = __ldg(&w->b2[0][lane]), bias1 = __ldg(&w->b2[1][lane]);
  float z[2][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    // ---- layer 1 (biases: W1 column 10 against the constant input) ----
    uint32_t a[4];
    ldsm_x4(xs + ((mt * 16 + r + 8 * (m & 1)) * kXStride + 8 * (m >> 1)) * 2, a[0], a[1], a[2], a[3]);
    float c1[4][4];
#pragma unroll
    for (int np = 0; np < 2; ++np) {
      const uint4 b = __ldg(&w->w1[np][lane]);
      mma16816_new(c1[2 * np], a[0], a[1], a[2], a[3], b.x, b.y);
      mma16816_new(c1[2 * np + 1], a[0], a[1], a[2], a[3], b.z, b.w);
    }
    uint32_t a2[2][4];
    acc_to_a(c1[0], c1[1], a2[0]);
    acc_to_a(c1[2], c1[3], a2[1]);
    // ---- layer 2 (biases as the first K-step's accumulator input) ----
    float c2[4][4];
#pragma unroll
    for (int np = 0; np < 2; ++np) {
      const uint4 b = __ldg(&w->w2[0][np][lane]);
      const float4 bias = np == 0 ? bias0 : bias1;
      mma16816_c(c2[2 * np], a2[0][0], a2[0][1], a2[0][2], a2[0][3], b.x, b.y, bias.x, bias.y);
      mma16816_c(c2[2 * np + 1], a2[0][0], a2[0][1], a2[0][2], a2[0][3], b.z, b.w, bias.z, bias.w);
    }
#pragma unroll
    for (int np = 0; np < 2; ++np) {
      const uint4 b = __ldg(&w->w2[1][np][lane]);
      mma16816(c2[2 * np], a2[1][0], a2[1][1], a2[1][2], a2[1][3], b.x, b.y);
      mma16816(c2[2 * np + 1], a2[1][0], a2[1][1], a2[1][2], a2[1][3], b.z, b.w);
    }
    uint32_t a3[2][4];
    acc_to_a(c2[0], c2[1], a3[0]);
    acc_to_a(c2[2], c2[3], a3[1]);
    // ---- layer 3 (column 0 of the N = 8 tile; b3 as the accumulator input) ----
    mma16816_c(z[mt], a3[0][0], a3[0][1], a3[0][2], a3[0][3], b3.x, b3.y, sc.b3, sc.b3);
    mma16816(z[mt], a3[1][0], a3[1][1], a3[1][2], a3[1][3], b3.z, b3.w);
  }
  // row rr of M-tile mt sits in lane 4 (rr % 8): register 0 for rr < 8, register 2 above
  const int src = 4 * (lane & 7);
  const float s00 = __shfl_sync(0xffffffffu, z[0][0], src);
  const float s02 = __shfl_sync(0xffffffffu, z[0][2], src);
  const float s10 = __shfl_sync(0xffffffffu, z[1][0], src);
  const float s12 = __shfl_sync(0xffffffffu, z[1][2], src);
  const float zz = lane < 8 ? s00 : lane < 16 ? s02 : lane < 24 ? s10 : s12;
  return sc.out_scale * softplus_fast(zz);
}

}  // namespace psl
