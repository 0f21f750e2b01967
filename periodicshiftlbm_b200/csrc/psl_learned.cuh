// The update kernels with the learned subgrid closure fused into the collision.
//
// Same per-cell work as step_kernel (applyLocalCellUpdate.h:1-74) except the relaxation
// rate: the cumulant collision's second-order central moments feed the per-cell MLP,
// whose eddy viscosity sets
//     omega = 1 / (3 (nu + nu_t) + 1/2)
// in place of the Smagorinsky rate of include/cellFunctions.h:157-198.  In the tcgen05
// kernel, a cell whose closure evaluation timed out (bounded wait) keeps the Smagorinsky
// rate.
//
// Two evaluations of the closure, one kernel each (same arithmetic around them):
//   step_learned_warp_kernel  per-warp tensor-core MMAs (psl_mlp_warp.cuh), the default;
//   step_learned_kernel       CTA-wide tcgen05 MMAs with TMEM accumulators (psl_mlp.cuh).
// Both run one 128-cell tile per CTA (the tcgen05 kernel stages its weights in shared memory
// and allocates and frees its 32 TMEM columns per CTA; the per-warp kernel reads its weights
// from global memory in fragment order, without a CTA barrier): a persistent loop
// over tiles made the compiler keep the 54 row offsets of the RowIndex in registers across
// iterations (120 registers against 72 for one tile per CTA).  Every thread takes part in
// its tile's MMAs (skip, solid and out-of-range cells with zero features), so the warp- or
// CTA-wide steps inside the closure are reached by all.
#pragma once
#include "psl_kernels.cuh"
#include "psl_mlp.cuh"
#include "psl_mlp_warp.cuh"

namespace psl {

template <typename S>
struct LearnedParams {
  RowIndex<S> ri;
  const uint8_t* marker;
  const float4* given;
  float4 given_uniform;
  RelaxationT<float> rx;    // Smagorinsky fallback
  const MlpDevice* mlp;      // tcgen05 layout
  const MlpFrag* mlpw;       // per-warp layout (fragment order, global memory)
  MlpScalars sc;             // normalisation, b3, output scale of the per-warp path
  float nu;                 // lattice viscosity of the grid
  float width;              // filter width fed to the closure (cell size / coarsest cell size)
  uint32_t n;
  unsigned int* health;
};

template <typename S>
__global__ void __launch_bounds__(kMlpRows) step_learned_kernel(const __grid_constant__ LearnedParams<S> p) {
  __shared__ MlpShared s;
  mlp_cta_setup(s, p.mlp);
  uint32_t phase = 0;
  {
    const uint32_t cell = blockIdx.x * kMlpRows + threadIdx.x;
    const uint8_t m = cell < p.n ? p.marker[cell] : make_marker(kSkip, 0);
    const int kind = marker_kind(m);
    float f[27];
    float K[3][3][3];
    float rho = 1.f, ux = 0.f, uy = 0.f, uz = 0.f, inv_rho = 1.f;
    float x[kMlpIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (kind != kSkip) {
      load_cell_ri<S>(p.ri, cell, f);
      if (kind == kSolid) {  // bounce-back: done before the closure, nothing to keep
#pragma unroll
        for (int q = 1; q < 27; q += 2) {
          const float t = f[q];
          f[q] = f[q + 1];
          f[q + 1] = t;
        }
        store_cell_ri<S>(p.ri, cell, f);
      } else {
        if (kind != kFluid) apply_boundary(m, f, p.given ? p.given[cell] : p.given_uniform);
        central_moments(f, K, rho, ux, uy, uz, inv_rho);
        mlp_features(K[2][0][0], K[0][2][0], K[0][0][2], K[1][1][0], K[1][0][1], K[0][1][1], rho, inv_rho, p.width, x);
      }
    }
    const float nu_t = mlp_eval(s, x, phase, p.health);
    if (kind != kSkip && kind != kSolid) {
      const float w = nu_t >= 0.f ? 1.f / (3.f * (p.nu + nu_t) + 0.5f) : smagorinsky_omega(K, rho, inv_rho, p.rx);
      relax_rebuild(f, K, rho, ux, uy, uz, inv_rho, w);
      if (p.health) {
        const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
        if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
      }
      store_cell_ri<S>(p.ri, cell, f);
    }
  }
  mlp_cta_teardown(s);
}

template <typename S>
__global__ void __launch_bounds__(kStepThreads, 7) step_learned_warp_kernel(const __grid_constant__ LearnedParams<S> p) {
  __shared__ __align__(16) __half xtile[kStepThreads / 32][32 * kXStride];
  __half* xt = xtile[threadIdx.x >> 5];
  {
    const uint32_t cell = blockIdx.x * kStepThreads + threadIdx.x;
    const uint8_t m = cell < p.n ? p.marker[cell] : make_marker(kSkip, 0);
    const int kind = marker_kind(m);
    float f[27];
    float K[3][3][3];
    float rho = 1.f, ux = 0.f, uy = 0.f, uz = 0.f, inv_rho = 1.f;
    float x[kMlpIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (kind != kSkip) {
      load_cell_ri<S>(p.ri, cell, f);
      if (kind == kSolid) {  // bounce-back: done before the closure, nothing to keep
#pragma unroll
        for (int q = 1; q < 27; q += 2) {
          const float t = f[q];
          f[q] = f[q + 1];
          f[q + 1] = t;
        }
        store_cell_ri<S>(p.ri, cell, f);
      } else {
        if (kind != kFluid) apply_boundary(m, f, p.given ? p.given[cell] : p.given_uniform);
        central_moments(f, K, rho, ux, uy, uz, inv_rho);
        mlp_features(K[2][0][0], K[0][2][0], K[0][0][2], K[1][1][0], K[1][0][1], K[0][1][1], rho, inv_rho, p.width, x);
      }
    }
    const float nu_t = mlp_warp_eval(p.mlpw, p.sc, xt, x);  // converges the warp first
    if (kind != kSkip && kind != kSolid) {
      relax_rebuild(f, K, rho, ux, uy, uz, inv_rho, 1.f / (3.f * (p.nu + nu_t) + 0.5f));
      if (p.health) {
        const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
        if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
      }
      store_cell_ri<S>(p.ri, cell, f);
    }
  }
}

// The closure alone on host-provided features (count x 10, raw), for parity tests of the
// tensor-core path: one thread per row, 128 rows per CTA.
static __global__ void __launch_bounds__(kMlpRows) mlp_infer_kernel(const MlpDevice* mlp, const float* features,
                                                                    int count, float* out, unsigned int* health) {
  __shared__ MlpShared s;
  mlp_cta_setup(s, mlp);
  uint32_t phase = 0;
  const int row = blockIdx.x * kMlpRows + threadIdx.x;
  float x[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i) x[i] = row < count ? features[(size_t)row * kMlpIn + i] : 0.f;
  const float nu_t = mlp_eval(s, x, phase, health);
  if (row < count) out[row] = nu_t;
  mlp_cta_teardown(s);
}

}  // namespace psl
