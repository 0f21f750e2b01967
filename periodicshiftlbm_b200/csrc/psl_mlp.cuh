// Per-cell MLP subgrid closure on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// The closure maps 10 features of a cell (6 non-equilibrium second moments, 3 invariants
// of that tensor, the filter width) through two hidden layers of 32 ReLU units to an
// eddy viscosity nu_t >= 0 (softplus output).  Weights are FP16, accumulation FP32.
//
// Mapping onto tcgen05: a CTA of 128 threads owns 128 cells, one per thread, so a layer is
// ONE M=128 MMA: A = the CTA's 128 feature (or activation) rows, staged in shared memory by
// the threads; B = the layer's weights (N x K, K-major) in shared memory; D = 128 TMEM
// lanes x N FP32 columns.  With the 32x32b TMEM load shape, warp w reads lanes 32w..32w+31,
// i.e. thread t of warp w receives exactly the row of its own cell: no shuffles.
//   layer 1: K=16 (10 features, zero padded) N=32
//   layer 2: K=32 (two K=16 MMAs)            N=32
//   layer 3: K=32 (two K=16 MMAs)            N=16 (row 0 of B3 holds the output weights)
// One thread issues the MMAs and commits them to an mbarrier; every wait on that mbarrier
// is bounded (on timeout the health word gets bit 2 and the cell falls back to
// Smagorinsky).
//
// Shared-memory operand layout (no swizzle, K-major "core matrix" layout of the tcgen05
// matrix descriptor): element (r, k) of an R-row operand lives at byte
//     (k / 8) * (R * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so 8 rows x 8 K-elements form one contiguous 128-byte core matrix; the descriptor's
// stride byte offset (between 8-row groups) is 128 and its leading byte offset (between
// 8-element K chunks) is R * 16.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace psl {

constexpr int kMlpIn = 10;
constexpr int kMlpHidden = 32;
constexpr int kMlpRows = 128;     // cells per CTA tile (the MMA's M)
constexpr int kMlpK1 = 16;        // padded input width
constexpr int kMlpN3 = 16;        // padded output width
constexpr int kMlpTmemCols = 32;  // TMEM columns a CTA allocates

// Byte offset of element (r, k) of an operand with `rows` rows in the layout above.
__host__ __device__ constexpr uint32_t mlp_operand_offset(uint32_t rows, uint32_t r, uint32_t k) {
  return (k / 8) * (rows * 16) + (r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
}

// The closure as the kernels read it: FP16 weights already in the operand layout, FP32
// biases and feature normalisation.
struct MlpDevice {
  __half w1[kMlpHidden * kMlpK1];      // 32 x 16  (1 KB)
  __half w2[kMlpHidden * kMlpHidden];  // 32 x 32  (2 KB)
  __half w3[kMlpN3 * kMlpHidden];      // 16 x 32  (1 KB)
  float b2[kMlpHidden];                // layer-1 biases ride in W1 column 10 (input 10 = 1)
  float b3;
  float out_scale;                     // nu_t = out_scale * softplus(z)
  float in_scale[kMlpIn];              // feature normalisation: x * in_scale + in_offset
  float in_offset[kMlpIn];
  float pad[2];
};
static_assert(sizeof(MlpDevice) % 16 == 0, "MlpDevice is copied in 16-byte units");

// Features of a cell from its second-order central moments (C_aa, C_ab), density and
// the filter width: Pi_neq = C - rho/3 I (per unit density), then trace, norm and
// det / |Pi|^2 of that tensor.
__device__ __forceinline__ void mlp_features(float c200, float c020, float c002, float c110, float c101, float c011,
                                             float rho, float inv_rho, float width, float (&x)[kMlpIn]) {
  const float third = rho * (1.f / 3.f);
  const float pxx = (c200 - third) * inv_rho, pyy = (c020 - third) * inv_rho, pzz = (c002 - third) * inv_rho;
  const float pxy = c110 * inv_rho, pxz = c101 * inv_rho, pyz = c011 * inv_rho;
  const float n2 = pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz);
  const float det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz);
  x[0] = pxx;
  x[1] = pyy;
  x[2] = pzz;
  x[3] = pxy;
  x[4] = pxz;
  x[5] = pyz;
  x[6] = pxx + pyy + pzz;
  x[7] = sqrtf(n2);
  x[8] = det / (n2 + 1e-30f);
  x[9] = width;
}

// ---- PTX wrappers --------------------------------------------------------------------
__device__ __forceinline__ uint32_t mlp_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: no swizzle, K-major, version 1 (sm_100).
__device__ __forceinline__ uint64_t mlp_smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(lbo_bytes >> 4) << 16) |
         ((uint64_t)(sbo_bytes >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: A = B = FP16, D = FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t mlp_idesc(uint32_t m, uint32_t n) {
  return (1u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mlp_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mlp_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mlp_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mlp_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void mlp_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mlp_mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the mbarrier phase with parity `parity` to complete; false on timeout.
__device__ __forceinline__ bool mlp_mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t spin = 0; spin < (1u << 22); ++spin) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mlp_tmem_alloc(uint32_t dst_smem, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void mlp_tmem_dealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void mlp_tmem_load16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float mlp_tmem_load1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  return __uint_as_float(r);
}

// ---- the CTA-wide closure evaluation -----------------------------------------------------
// Shared state of one CTA (declared by the kernel, 16-byte aligned operand buffers).
struct MlpShared {
  __align__(128) unsigned char a1[kMlpRows * kMlpK1 * 2];      // 4 KB  features, FP16
  __align__(128) unsigned char a2[kMlpRows * kMlpHidden * 2];  // 8 KB  activations, FP16
  __align__(128) MlpDevice w;                                   // weights + biases
  __align__(8) unsigned long long mbar;
  uint32_t tmem;
  uint32_t phase;   // parity of the next mbarrier completion
  int failed;       // a wait timed out: the closure is off for the rest of the launch
};

// Copy the closure into shared memory (all threads), set up the mbarrier (thread 0) and
// allocate TMEM (warp 0).  Ends with a CTA barrier.
__device__ __forceinline__ void mlp_cta_setup(MlpShared& s, const MlpDevice* __restrict__ w) {
  const int4* src = reinterpret_cast<const int4*>(w);
  int4* dst = reinterpret_cast<int4*>(&s.w);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpDevice) / 16); i += blockDim.x) dst[i] = src[i];
  if (threadIdx.x == 0) {
    mlp_mbar_init(mlp_smem_u32(&s.mbar));
    s.phase = 0;
    s.failed = 0;
  }
  if (threadIdx.x < 32) mlp_tmem_alloc(mlp_smem_u32(&s.tmem), kMlpTmemCols);
  mlp_fence_before();
  __syncthreads();
  mlp_fence_after();
}

// Frees the TMEM columns.  After a timed-out wait, first waits (bounded) for the MMAs
// still in flight so the columns are not released under them.
__device__ __forceinline__ void mlp_cta_teardown(MlpShared& s) {
  mlp_fence_before();
  __syncthreads();
  mlp_fence_after();
  if (s.failed && threadIdx.x == 0) {
    const uint32_t mbar = mlp_smem_u32(&s.mbar);
    for (int k = 0; k < 3; ++k) mlp_mbar_wait(mbar, (s.phase + k) & 1u);
  }
  __syncthreads();
  if (threadIdx.x < 32) mlp_tmem_dealloc(s.tmem, kMlpTmemCols);
}

// Evaluate the closure for the CTA's 128 cells; every thread of the CTA must call it (the
// thread's row is threadIdx.x).  `x` holds the thread's raw features.  Returns nu_t, or a
// negative value when the closure is unavailable (a wait timed out in this launch; the
// caller falls back to Smagorinsky).  `phase` is the CTA's running mbarrier parity (every
// thread keeps its own copy; three completions per call).
__device__ __forceinline__ float mlp_eval(MlpShared& s, const float (&x)[kMlpIn], uint32_t& phase,
                                          unsigned int* health) {
  const uint32_t row = threadIdx.x;
  const uint32_t warp_lane0 = (threadIdx.x & ~31u) << 16;  // TMEM lane field of this warp
  const uint32_t mbar = mlp_smem_u32(&s.mbar);
  const uint32_t t_d = s.tmem;
  // ---- layer 1 operand: normalised features, FP16, K padded to 16 ----
  {
    float xn[16];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) xn[i] = fmaf(x[i], s.w.in_scale[i], s.w.in_offset[i]);
    xn[kMlpIn] = 1.f;  // carries the layer-1 biases (W1 column 10)
#pragma unroll
    for (int i = kMlpIn + 1; i < 16; ++i) xn[i] = 0.f;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      __half2 h[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) h[e] = __floats2half2_rn(xn[c * 8 + 2 * e], xn[c * 8 + 2 * e + 1]);
      *reinterpret_cast<uint4*>(s.a1 + mlp_operand_offset(kMlpRows, row, c * 8)) = *reinterpret_cast<uint4*>(h);
    }
  }
  bool ok = !s.failed;
  // three layers; A of layer 1 is a1, of layers 2 and 3 a2
#pragma unroll
  for (int layer = 0; layer < 3; ++layer) {
    mlp_proxy_fence();
    mlp_fence_before();
    __syncthreads();
    mlp_fence_after();
    if (threadIdx.x == 0 && ok) {
      const uint32_t a_base = mlp_smem_u32(layer == 0 ? s.a1 : s.a2);
      const uint32_t b_base = mlp_smem_u32(layer == 0 ? (const void*)s.w.w1 : (layer == 1 ? (const void*)s.w.w2 : (const void*)s.w.w3));
      const uint32_t b_rows = layer == 2 ? kMlpN3 : kMlpHidden;
      const uint32_t idesc = mlp_idesc(kMlpRows, b_rows);
      const int ksteps = layer == 0 ? 1 : 2;
      for (int kk = 0; kk < ksteps; ++kk) {
        // a K=16 step spans two 8-element chunks: advance by two leading byte offsets
        const uint64_t ad = mlp_smem_desc(a_base + kk * 2 * (kMlpRows * 16), kMlpRows * 16, 128);
        const uint64_t bd = mlp_smem_desc(b_base + kk * 2 * (b_rows * 16), b_rows * 16, 128);
        mlp_mma(t_d, ad, bd, idesc, kk > 0 ? 1u : 0u);
      }
      mlp_commit(mbar);
    }
    // (after a failure nothing more is issued: `ok` is CTA-uniform, read after a barrier)
    if (ok) {
      const bool done = mlp_mbar_wait(mbar, phase);
      phase ^= 1u;
      if (!done) {
        ok = false;
        s.failed = 1;
        if (threadIdx.x == 0) s.phase = phase;
        if (health) atomicOr(health, 4u);
      }
    }
    mlp_fence_after();
    if (layer < 2) {
      // bias + ReLU, FP16, into a2 (16 columns at a time).  The next layer's MMA reads a2
      // only after every thread's row is written (barrier at the top of the loop); a2 is
      // free: the MMA that read it has completed.
      const float* b = layer == 0 ? nullptr : s.w.b2;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        float h[16];
        mlp_tmem_load16(t_d + warp_lane0 + half * 16, h);
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          __half2 hv[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int i = c * 8 + 2 * e;
            const float bi = b ? b[half * 16 + i] : 0.f, bj = b ? b[half * 16 + i + 1] : 0.f;
            hv[e] = __hmax2(__floats2half2_rn(h[i] + bi, h[i + 1] + bj), __float2half2_rn(0.f));
          }
          *reinterpret_cast<uint4*>(s.a2 + mlp_operand_offset(kMlpRows, row, half * 16 + c * 8)) =
              *reinterpret_cast<uint4*>(hv);
        }
      }
    }
  }
  const float z = mlp_tmem_load1(t_d + warp_lane0) + s.w.b3;
  const float sp = z > 20.f ? z : log1pf(__expf(z));
  return ok ? s.w.out_scale * sp : -1.f;
}

}  // namespace psl
