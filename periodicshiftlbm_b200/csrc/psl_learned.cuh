// The update kernels with the learned subgrid closure fused into the collision.
//
// Same per-cell work as the plain update (applyLocalCellUpdate.h:1-74) except the
// relaxation rate: the cell's second-order central moments feed the per-cell MLP, whose
// eddy viscosity sets
//     omega = 1 / (3 (nu + nu_t) + 1/2)
// in place of the Smagorinsky rate of include/cellFunctions.h:157-198.
//
// The closure is evaluated per warp with tensor-core MMAs (psl_mlp_warp.cuh) inside the
// update kernel (step_learned_warp_kernel, one thread per cell): 16-bit storage collides on
// g = f - w (psl_collision_g.cuh), FP32 in the plain FP32 update's operation order.  Every
// thread takes part in its warp's MMAs (skip, solid and out-of-range cells with zero
// features), so the warp-wide steps inside the closure are reached by all lanes.  The
// CTA-wide tcgen05 evaluation (psl_mlp.cuh) serves the closure's batched inference.
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
  const MlpFrag* mlpw;       // fragment order, global memory
  MlpScalars sc;             // normalisation, b3, output scale
  float nu;                 // lattice viscosity of the grid
  float width;              // filter width fed to the closure (cell size / coarsest cell size)
  uint32_t n;
  unsigned int* health;
  uint32_t rot;              // thread-to-cell rotation (cell_of_thread)
  uint16_t* nut;             // kStoreNu: each collided cell's nu_t as FP16, held for the updates
                             // until the next evaluation (step_kernel_g, kRateNuField)
  ThreadRange range;         // the threads of cell_of_thread this launch runs
};

// The closure's features from D = C - rho/3 I (the g-form moments): the same quantities
// as mlp_features (Pi_neq = D / rho, its trace, norm and det / |Pi|^2, the filter width),
// with the single-instruction square root and reciprocal of the g-form collision (the
// features enter the network as FP16).
__device__ __forceinline__ void mlp_features_d(const CellMomentsG& m, float width, float (&x)[kMlpIn]) {
  const float r = m.inv_rho;
  const float pxx = m.dxx * r, pyy = m.dyy * r, pzz = m.dzz * r;
  const float pxy = m.dxy * r, pxz = m.dxz * r, pyz = m.dyz * r;
  const float n2 = pxx * pxx + pyy * pyy + pzz * pzz + 2.f * (pxy * pxy + pxz * pxz + pyz * pyz);
  const float det = pxx * (pyy * pzz - pyz * pyz) - pxy * (pxy * pzz - pyz * pxz) + pxz * (pxy * pyz - pyy * pxz);
  x[0] = pxx;
  x[1] = pyy;
  x[2] = pzz;
  x[3] = pxy;
  x[4] = pxz;
  x[5] = pyz;
  x[6] = pxx + pyy + pzz;
  x[7] = gsqrt(n2);
  x[8] = det * grecip(n2 + 1e-30f);
  x[9] = width;
}

// One thread per cell with the fused closure.  16-bit storage collides on its stored
// g = f - w (only the ten moments live across the closure's MMAs), fluid cells starting the
// moment sums from the stored bits; FP32 runs the plain FP32 update's operation order, only
// the rate differs.  kFlat: rows mapped twice, addressed without the wrap.
template <typename A, bool kFlat, typename S>
__device__ __forceinline__ void load_rows(const RowIndex<S>& r, uint32_t cell, typename A::calc (&f)[27]) {
  if constexpr (kFlat) load_cell_flat<A>(r, cell, f);
  else load_cell_as<A>(r, cell, f);
}
template <typename A, bool kFlat, typename S>
__device__ __forceinline__ void store_rows(const RowIndex<S>& r, uint32_t cell, const typename A::calc (&f)[27]) {
  if constexpr (kFlat) store_cell_flat<A>(r, cell, f);
  else store_cell_as<A>(r, cell, f);
}

// 7 blocks of 128 per SM (72 registers; ptxas keeps ~40 bytes in local memory, L1-resident):
// 1.2% faster than 6 blocks at 80 registers without spills, measured on the sphere case.
template <typename S, bool kFlat, bool kStoreNu>
__global__ void __launch_bounds__(kStepThreads, 7) step_learned_warp_kernel(const __grid_constant__ LearnedParams<S> p) {
  static_assert(!kStoreNu || kCollidesOnG<S>, "the held nu_t field serves the 16-bit update only");
  __shared__ __align__(16) float bc_slot[kStepThreads][27];
  // the warp's FP16 feature tile lives in its own lanes' boundary slots (free after the
  // __syncwarp that follows every lane's boundary condition)
  __half* xt = reinterpret_cast<__half*>(&bc_slot[threadIdx.x & ~31u][0]);
  const uint32_t u = blockIdx.x * kStepThreads + threadIdx.x;
  const bool in = u < p.range.count;
  const uint32_t cell = in ? cell_of_thread(range_thread(p.range, u), p.rot, p.n) : 0u;
  const uint8_t m = in ? p.marker[cell] : make_marker(kSkip, 0);
  const int kind = marker_kind(m);
  float x[kMlpIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float f[27];
  const bool collides = kind != kSkip && kind != kSolid;
  if constexpr (kCollidesOnG<S>) {
    using B = StoredBits<S>;
    uint16_t h[27];
    if (kind == kSolid) {  // bounce-back: done before the closure, nothing to keep
      load_rows<B, kFlat>(p.ri, cell, h);
#pragma unroll
      for (int q = 1; q < 27; q += 2) {
        const uint16_t t = h[q];
        h[q] = h[q + 1];
        h[q + 1] = t;
      }
      store_rows<B, kFlat>(p.ri, cell, h);
    }
    if (collides) load_rows<B, kFlat>(p.ri, cell, h);
    CellMomentsG cm{};
    const bool bc = collides && kind != kFluid;
    if (!__any_sync(0xffffffffu, bc)) {
      if (collides) cm = cell_moments_from_raw(raw_moments_g_bits<S::kind == kStoreBF16>(h));
    } else if (collides) {
      // a warp holding boundary cells sums every lane's moments from converted values (the
      // same bits as from the stored bits)
#pragma unroll
      for (int q = 0; q < 27; ++q) f[q] = B::to_float(h[q]);
      if (bc) {
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] += lattice_weight(q);
        apply_boundary_at(m, f, p.given ? p.given[cell] : p.given_uniform, bc_slot[threadIdx.x]);
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] -= lattice_weight(q);
      }
      cm = cell_moments_g(f);
    }
    if (collides) {
      if (p.health && !finite_density(cm.rho)) atomicOr(p.health, 1u);
      mlp_features_d(cm, p.width, x);
    }
    __syncwarp();
    const float nu_t = mlp_warp_eval(p.mlpw, p.sc, xt, x);
    if (collides) {
      if constexpr (kStoreNu) p.nut[cell] = __half_as_ushort(__float2half_rn(nu_t));
      relax_rebuild_g(f, cm, grecip(3.f * (p.nu + nu_t) + 0.5f));
      store_rows<StoredOf<S>, kFlat>(p.ri, cell, f);
    }
  } else {
    using A = StoredOf<S>;
    if (kind == kSolid) {  // bounce-back: done before the closure, nothing to keep
      load_rows<A, kFlat>(p.ri, cell, f);
#pragma unroll
      for (int q = 1; q < 27; q += 2) {
        const float t = f[q];
        f[q] = f[q + 1];
        f[q + 1] = t;
      }
      store_rows<A, kFlat>(p.ri, cell, f);
    }
    if (collides) load_rows<A, kFlat>(p.ri, cell, f);
    float K[3][3][3];
    float rho = 1.f, ux = 0.f, uy = 0.f, uz = 0.f, inv_rho = 1.f;
    if (collides) {
      if (kind != kFluid) apply_boundary_at(m, f, p.given ? p.given[cell] : p.given_uniform, bc_slot[threadIdx.x]);
      central_moments(f, K, rho, ux, uy, uz, inv_rho);
      mlp_features(K[2][0][0], K[0][2][0], K[0][0][2], K[1][1][0], K[1][0][1], K[0][1][1], rho, inv_rho, p.width, x);
    }
    __syncwarp();
    const float nu_t = mlp_warp_eval(p.mlpw, p.sc, xt, x);
    if (collides) {
      relax_rebuild(f, K, rho, ux, uy, uz, inv_rho, 1.f / (3.f * (p.nu + nu_t) + 0.5f));
      if (p.health) {
        const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
        if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
      }
      store_rows<A, kFlat>(p.ri, cell, f);
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
