// CUDA kernels of the per-step lattice update (sm_100a).
//
// Data layout in HBM (per grid): populations as 27 rows of `stride` elements (structure of
// arrays, the reference's fArray[27][N], include/types.h:42-45), row q starting 128-byte
// aligned; a one-byte marker per cell; 27 periodic-shift offsets kept on the host and
// passed as kernel parameters.  Population q of cell c lives at row q, address
// (c + shift_q) mod N (applyStreaming.h:33-41); streaming only changes the 27 offsets.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "psl_bc_generated.cuh"
#include "psl_collision.cuh"
#include "psl_collision_g.cuh"
#include "psl_hooks.cuh"
#include "psl_lattice.cuh"
#include "psl_storage.cuh"

namespace psl {

constexpr int kStepThreads = 128;

// Shifted address of population q of `cell` (getShiftedIndex, applyStreaming.h:33-41).
// cell < n and shift < n, so one conditional subtraction wraps it.
__device__ __forceinline__ uint32_t shifted(uint32_t cell, uint32_t shift, uint32_t n) {
  const uint32_t a = cell + shift;
  return a >= n ? a - n : a;
}

template <typename S>
struct GridView {
  typename S::type* fq[27];  // row q of the population array
  uint32_t shift[27];
  uint32_t n;                // cells (the periodic-shift modulus)
};

// ------------------------------------------------------------------------------------------
// fused per-cell update: gather -> bounce-back | (boundary condition) -> collision -> scatter
// ------------------------------------------------------------------------------------------
// Row addressing for the update kernel: one base pointer and 32-bit per-population
// offsets.  Population q of `cell` lives at base[off_q + cell] while cell < lim_q, else at
// base[off_q + cell - N], with off_q = q*stride + shift_q and lim_q = N - shift_q.  32-bit
// kernel parameters serve as constant-bank operands, so no per-population 64-bit pointer
// has to be fetched; usable while 27*stride + N < 2^32.
template <typename S>
struct RowIndex {
  typename S::type* base;
  uint32_t off[27];
  uint32_t lim[27];
  uint32_t n;
};


// The threads of an update launch: launch thread u (u < count) is thread
// t_begin + u + (u >= gap_at ? gap_len : 0) of cell_of_thread, so one launch can run a
// contiguous range of threads, or all threads but one contiguous range.
struct ThreadRange {
  uint32_t t_begin, gap_at, gap_len, count;
};
__host__ __device__ inline ThreadRange full_range(uint32_t n) { return ThreadRange{0u, 0xffffffffu, 0u, n}; }
__device__ __forceinline__ uint32_t range_thread(const ThreadRange& r, uint32_t u) {
  return r.t_begin + u + (u >= r.gap_at ? r.gap_len : 0u);
}

template <typename S>
struct StepParams {
  GridView<S> g;
  RowIndex<S> ri;
  const uint8_t* marker;
  const float4* given;   // per-cell (rho, ux, uy, uz) for boundary cells, or null
  float4 given_uniform;  // used when `given` is null
  const float* cs;       // per-cell Smagorinsky constant (getSmagorinskyConstant), or null: rx.cs18
  RelaxationT<typename S::calc> rx;
  unsigned int* health;  // bit 0 set when a collided cell's density is not finite/positive
  uint32_t rot;          // thread-to-cell rotation (cell_of_thread)
  const uint16_t* nut;   // per-cell FP16 eddy viscosity held from the learned closure's last
                         // evaluation (kRateNuField), or null
  float nu;              // the grid's lattice viscosity (kRateNuField)
  ThreadRange range;     // the threads of cell_of_thread this launch runs
};

// Relaxation rate of the 16-bit update kernel:
//   kRateUniform   Smagorinsky with the grid's constant
//   kRateCsField   Smagorinsky with the cell's constant (p.cs)
//   kRateNuField   omega = 1 / (3 (nu + nu_t) + 1/2) with the cell's held nu_t (p.nut), the
//                  learned closure's rate between two of its evaluations
enum RateKind : int { kRateUniform = 0, kRateCsField = 1, kRateNuField = 2 };

// Cell of thread t: t - rot, cyclically.  With rot = 16 and Nx a multiple of 32, the last
// cell of one x-row and the first of the next (both x-face cells, i = Nx - 1 and i = 0) fall
// into the same warp, so only one warp in Nx / 32 carries the boundary branch instead of two
// (every cell still updated once; the warps still cover 32 consecutive cells).
__device__ __forceinline__ uint32_t cell_of_thread(uint32_t t, uint32_t rot, uint32_t n) {
  return t >= rot ? t - rot : t + n - rot;
}

// The relaxation parameters of one cell: the grid's, with the cell's own Smagorinsky
// constant when the grid has a per-cell field.
template <typename T>
__device__ __forceinline__ RelaxationT<T> cell_relaxation(const RelaxationT<T>& rx, const float* cs, uint32_t cell) {
  RelaxationT<T> r = rx;
  if (cs) r.cs18 = T(18) * T(cs[cell]);
  return r;
}

// The boundary branch runs for ~2% of cells; keeping it out of line keeps the hot path's
// instruction footprint small.  (applyLocalCellUpdate.h:41-67)
template <typename T>
static __device__ __noinline__ void apply_boundary_out_of_line(uint8_t m, T* populations, float4 given) {
  T (&f)[27] = *reinterpret_cast<T(*)[27]>(populations);
  const int kind = marker_kind(m), normal = marker_normal(m);
  T rho = given.x, ux = given.y, uy = given.z, uz = given.w;
  if (kind == kMirror) {
    bc::mirror(normal, f);
    return;
  }
  if (kind == kGivenRho) bc::restore_u(normal, f, rho, ux, uy, uz);
  else if (kind == kGivenU) bc::restore_rho(normal, f, rho, ux, uy, uz);
  else if (kind == kGivenNone) bc::restore_rho_u(normal, f, rho, ux, uy, uz);
  bc::mbbc(normal, f, rho, ux, uy, uz);
}

// The call site: the populations go through the thread's own slot in shared memory,
// written and read inside the boundary branch only.  Passing the caller's array by
// reference would take its address, and nvcc then keeps it in local memory for every cell
// (a stack write of all 27 populations per fluid cell too); a copy in local memory inside
// the branch still cost a warp holding one inflow cell 8% of the update launch on a
// 512-wide grid, the shared-memory slot 3%.
template <typename T>
__device__ __forceinline__ void apply_boundary_at(uint8_t m, T (&f)[27], float4 given, T* mine) {
#pragma unroll
  for (int q = 0; q < 27; ++q) mine[q] = f[q];
  apply_boundary_out_of_line(m, mine, given);
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = mine[q];
}
// ... with a kernel-wide slot array of kSlots >= the block's threads.
template <int kSlots = kStepThreads, typename T>
__device__ __forceinline__ void apply_boundary(uint8_t m, T (&f)[27], float4 given) {
  __shared__ T slot[kSlots][27];
  apply_boundary_at(m, f, given, slot[threadIdx.x]);
}

// The collided-cell body of the 16-bit forms on the stored deviations g = f - w: the
// boundary functions work on f (g + w, then back), the collision on g (psl_collision_g.cuh).
// Shared by the one-cell and the batched update, so both give the same bits.
__device__ __forceinline__ void collide_cell_g(int kind, uint8_t m, float (&g)[27], const float4* given,
                                               float4 given_uniform, uint32_t cell, const RelaxationT<float>& rx,
                                               float cs18, unsigned int* health, float* slot) {
  if (kind != kFluid) {
#pragma unroll
    for (int q = 0; q < 27; ++q) g[q] += lattice_weight(q);
    apply_boundary_at(m, g, given ? given[cell] : given_uniform, slot);
#pragma unroll
    for (int q = 0; q < 27; ++q) g[q] -= lattice_weight(q);
  }
  const CellMomentsG cm = cell_moments_g(g);
  if (health && !finite_density(cm.rho)) atomicOr(health, 1u);
  relax_rebuild_g(g, cm, smagorinsky_omega_g(cm, rx.omega0, rx.tau, rx.tau2, cs18));
}

// Gathers / scatters of one cell through accessor A (S itself, or StoredOf<S> for the
// stored values): GridView (64-bit row pointers) or RowIndex (base + 32-bit offsets).
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void load_cell_as(const GridView<S>& g, uint32_t cell, typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    f[Q] = A::template load<Q>(g.fq[Q] + shifted(cell, g.shift[Q], g.n));
    load_cell_as<A, S, Q + 1>(g, cell, f);
  }
}
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void store_cell_as(const GridView<S>& g, uint32_t cell, const typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    A::template store<Q>(g.fq[Q] + shifted(cell, g.shift[Q], g.n), f[Q]);
    store_cell_as<A, S, Q + 1>(g, cell, f);
  }
}
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void load_cell_as(const RowIndex<S>& r, uint32_t cell, typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    uint32_t i = cell + r.off[Q];
    if (cell >= r.lim[Q]) i -= r.n;
    f[Q] = A::template load_once<Q>(r.base + i);
    load_cell_as<A, S, Q + 1>(r, cell, f);
  }
}
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void store_cell_as(const RowIndex<S>& r, uint32_t cell, const typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    uint32_t i = cell + r.off[Q];
    if (cell >= r.lim[Q]) i -= r.n;
    A::template store_once<Q>(r.base + i, f[Q]);
    store_cell_as<A, S, Q + 1>(r, cell, f);
  }
}
template <typename S>
__device__ __forceinline__ void load_cell(const GridView<S>& g, uint32_t cell, typename S::calc (&f)[27]) {
  load_cell_as<S>(g, cell, f);
}
template <typename S>
__device__ __forceinline__ void store_cell(const GridView<S>& g, uint32_t cell, const typename S::calc (&f)[27]) {
  store_cell_as<S>(g, cell, f);
}
// Rows mapped twice (psl_rowmap.cu): cell + off_q < row start + 2N addresses the wrapped
// element through the row's second mapping, so no wrap compare.
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void load_cell_flat(const RowIndex<S>& r, uint32_t cell, typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    f[Q] = A::template load_once<Q>(r.base + (cell + r.off[Q]));
    load_cell_flat<A, S, Q + 1>(r, cell, f);
  }
}
template <typename A, typename S, int Q = 0>
__device__ __forceinline__ void store_cell_flat(const RowIndex<S>& r, uint32_t cell, const typename A::calc (&f)[27]) {
  if constexpr (Q < 27) {
    A::template store_once<Q>(r.base + (cell + r.off[Q]), f[Q]);
    store_cell_flat<A, S, Q + 1>(r, cell, f);
  }
}
template <typename S>
__device__ __forceinline__ void load_cell_ri(const RowIndex<S>& r, uint32_t cell, typename S::calc (&f)[27]) {
  load_cell_as<S>(r, cell, f);
}
template <typename S>
__device__ __forceinline__ void store_cell_ri(const RowIndex<S>& r, uint32_t cell, const typename S::calc (&f)[27]) {
  store_cell_as<S>(r, cell, f);
}


// The per-cell body (applyLocalCellUpdate.h:21-72): bounce-back for solid cells; for the
// others the boundary condition of the marker, the collision and a density health check.
template <int kSlots = kStepThreads, typename T>
__device__ __forceinline__ void local_cell_update(int kind, uint8_t m, T (&f)[27], const float4* given, float4 given_uniform,
                                                  uint32_t cell, const RelaxationT<T>& rx, unsigned int* health) {
  if (kind == kSolid) {
#pragma unroll
    for (int q = 1; q < 27; q += 2) {
      const T t = f[q];
      f[q] = f[q + 1];
      f[q + 1] = t;
    }
  } else {
    if (kind != kFluid) apply_boundary<kSlots>(m, f, given ? given[cell] : given_uniform);
    collide<false>(f, rx);
    if (health) {
      const T r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
      if (!(r > T(0) && r < T(1.0e30))) atomicOr(health, 1u);
    }
  }
}

// Population addressing of the update kernels:
//   kAddrView   64-bit row pointers with the periodic wrap (GridView)
//   kAddrIndex  base + 32-bit row offsets with the wrap (RowIndex; 27 rows + N < 2^32 elements)
//   kAddrFlat   base + 32-bit row offsets without the wrap, on rows mapped twice
enum RowAddr : int { kAddrView = 0, kAddrIndex = 1, kAddrFlat = 2 };

template <typename A, int kAddr, typename S>
__device__ __forceinline__ void load_for(const StepParams<S>& p, uint32_t cell, typename A::calc (&f)[27]) {
  if constexpr (kAddr == kAddrFlat) load_cell_flat<A>(p.ri, cell, f);
  else if constexpr (kAddr == kAddrIndex) load_cell_as<A>(p.ri, cell, f);
  else load_cell_as<A>(p.g, cell, f);
}
template <typename A, int kAddr, typename S>
__device__ __forceinline__ void store_for(const StepParams<S>& p, uint32_t cell, const typename A::calc (&f)[27]) {
  if constexpr (kAddr == kAddrFlat) store_cell_flat<A>(p.ri, cell, f);
  else if constexpr (kAddr == kAddrIndex) store_cell_as<A>(p.ri, cell, f);
  else store_cell_as<A>(p.g, cell, f);
}
// The update of one cell (applyLocalCellUpdate.h:21-72) for FP32 and FP64 storage:
// collide<false> on f, the reference's operation order.
template <typename S, int kAddr>
__device__ __forceinline__ void update_one_cell(const StepParams<S>& p, uint32_t cell, uint8_t m) {
  const int kind = marker_kind(m);
  if (kind == kSkip) return;
  using T = typename S::calc;
  T f[27];
  load_for<StoredOf<S>, kAddr>(p, cell, f);
  if (kind == kSolid) {
#pragma unroll
    for (int q = 1; q < 27; q += 2) {
      const T t = f[q];
      f[q] = f[q + 1];
      f[q + 1] = t;
    }
  } else {
    if (kind != kFluid) apply_boundary(m, f, p.given ? p.given[cell] : p.given_uniform);
    collide<false>(f, cell_relaxation(p.rx, p.cs, cell));
    if (p.health) {
      const T r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
      if (!(r > T(0) && r < T(1.0e30))) atomicOr(p.health, 1u);
    }
  }
  store_for<StoredOf<S>, kAddr>(p, cell, f);
}

// The same for the 16-bit forms, on their stored bits g = f - w (applyLocalCellUpdate.h:
// 21-72): solid cells swap the bits; fluid cells start the moment sums from them
// (raw_moments_g_bits); boundary cells go through f = g + w for the boundary functions; all
// collide on g (psl_collision_g.cuh), bitwise as collide_cell_g on the converted values.
// `slot`: the thread's shared-memory slot for the boundary functions.  All 32 lanes of the
// warp call it together (the boundary test is warp-wide).  Written for the register
// allocator: the loads and the collision run on every lane and only the stores are
// predicated, instead of early returns (which cost ~50 spilled registers at the 64-register
// cap).  `cell` must be < N.
template <typename S, int kAddr, int kRate>
__device__ __forceinline__ void update_one_cell_g(const StepParams<S>& p, uint32_t cell, uint8_t m, float* slot) {
  using B = StoredBits<S>;
  const int kind = marker_kind(m);
  uint16_t h[27];
  if (kind == kSolid) {  // bounce-back: g and f swap alike (w_q = w_opposite(q))
    load_for<B, kAddr>(p, cell, h);
#pragma unroll
    for (int q = 1; q < 27; q += 2) {
      const uint16_t t = h[q];
      h[q] = h[q + 1];
      h[q + 1] = t;
    }
    store_for<B, kAddr>(p, cell, h);
  }
  // every lane loads (a lane that does not collide -- a skipped cell in a mixed warp, a lane
  // past the grid on cell 0 -- computes on real values and stores nothing): cheaper than
  // predicating the loads and zeroing the rest
  load_for<B, kAddr>(p, cell, h);
  // the kept nu_t, loaded with the populations (every lane: cell < N)
  const uint16_t nut_bits = kRate == kRateNuField ? __ldg(p.nut + cell) : (uint16_t)0;
  const bool collides = kind != kSkip && kind != kSolid;
  float g[27];
  CellMomentsG cm;
  const bool bc = collides && kind != kFluid;
  if (!__any_sync(0xffffffffu, bc)) {
    cm = cell_moments_from_raw(raw_moments_g_bits<S::kind == kStoreBF16>(h));
  } else {
    // a warp holding boundary cells sums every lane's moments from converted values (the
    // same bits as from the stored bits), so its fluid lanes do not run a second sum
#pragma unroll
    for (int q = 0; q < 27; ++q) g[q] = B::to_float(h[q]);
    if (bc) {
#pragma unroll
      for (int q = 0; q < 27; ++q) g[q] += lattice_weight(q);
      apply_boundary_at(m, g, p.given ? p.given[cell] : p.given_uniform, slot);
#pragma unroll
      for (int q = 0; q < 27; ++q) g[q] -= lattice_weight(q);
    }
    cm = cell_moments_g(g);
  }
  if (collides && p.health && !finite_density(cm.rho)) atomicOr(p.health, 1u);
  float omega;
  if constexpr (kRate == kRateNuField) {
    const float nu_t = __half2float(__ushort_as_half(nut_bits));
    omega = grecip(3.f * (p.nu + nu_t) + 0.5f);  // the learned closure's expression (psl_learned.cuh)
  } else {
    const float cs18 = kRate == kRateCsField && collides ? 18.f * p.cs[cell] : p.rx.cs18;
    omega = smagorinsky_omega_g(cm, p.rx.omega0, p.rx.tau, p.rx.tau2, cs18);
  }
  relax_rebuild_g(g, cm, omega);
  if (collides) store_for<StoredOf<S>, kAddr>(p, cell, g);
}

// One thread per cell: FP32 / FP64 storage.
template <typename S, int kAddr>
__global__ void __launch_bounds__(kStepThreads) step_kernel(const __grid_constant__ StepParams<S> p) {
  static_assert(!kCollidesOnG<S>, "16-bit storage runs step_kernel_g");
  const uint32_t u = blockIdx.x * kStepThreads + threadIdx.x;
  if (u >= p.range.count) return;
  const uint32_t cell = cell_of_thread(range_thread(p.range, u), p.rot, p.g.n);
  update_one_cell<S, kAddr>(p, cell, p.marker[cell]);
}

// One thread per cell: the 16-bit forms, held to 64 registers (8 blocks of 128 per SM;
// 4 with 64-bit row pointers).  Left free the compiler hoists loads into 96 registers and
// the lower occupancy costs more than the hoisting gains.
// kRate: where the relaxation rate comes from (RateKind).
template <typename S, int kAddr, int kRate>
__global__ void __launch_bounds__(kStepThreads, kAddr == kAddrView ? 4 : 8) step_kernel_g(const __grid_constant__ StepParams<S> p) {
  static_assert(kCollidesOnG<S>, "FP32 / FP64 storage runs step_kernel");
  __shared__ float slot[kStepThreads][27];
  const uint32_t u = blockIdx.x * kStepThreads + threadIdx.x;
  const bool in = u < p.range.count;
  const uint32_t cell = in ? cell_of_thread(range_thread(p.range, u), p.rot, p.g.n) : 0u;
  const uint8_t m = in ? p.marker[cell] : make_marker(kSkip, 0);
  if (__all_sync(0xffffffffu, marker_kind(m) == kSkip)) return;  // ghost layers, refined interior
  update_one_cell_g<S, kAddr, kRate>(p, cell, m, slot[threadIdx.x]);
}

// ------------------------------------------------------------------------------------------
// customised update: moving walls, forced-velocity cells, body force
// ------------------------------------------------------------------------------------------
// applyMovingBounceback (include/boundaryConditions/applyMovingBounceback.h:8-60): the
// opposite pair (q, q+1) swaps and picks up -/+ 6 w_q (c_q . u_wall); the products are
// rounded separately from the additions, as the reference's host build does.
__device__ __forceinline__ void moving_bounceback(float (&f)[27], float ux, float uy, float uz) {
#pragma unroll
  for (int q = 1; q < 27; q += 2) {
    const float w6 = q <= 6 ? 4.0f / 9.0f : (q <= 18 ? 1.0f / 9.0f : 1.0f / 36.0f);
    float cu = cx(q) != 0 ? (cx(q) > 0 ? ux : -ux) : 0.f;  // c_q . u in the reference's order
    if (cy(q) != 0) cu = cx(q) != 0 ? (cy(q) > 0 ? cu + uy : cu - uy) : (cy(q) > 0 ? uy : -uy);
    if (cz(q) != 0) cu = (cx(q) != 0 || cy(q) != 0) ? (cz(q) > 0 ? cu + uz : cu - uz) : (cz(q) > 0 ? uz : -uz);
    const float d = __fmul_rn(w6, cu);
    const float t = f[q];
    f[q] = __fadd_rn(f[q + 1], d);
    f[q + 1] = __fsub_rn(t, d);
  }
}

template <typename S>
struct CustomParams {
  StepParams<S> base;
  float3 body;  // uniform body force on every collided cell (lattice units)
};

// The update of a customised case (the pattern of M35Full/applyLocalCellUpdateCustomized.h
// and M40Impeller/applyLocalCellUpdateCustomized.h on PS grids):
//   solid cell, marker normal 1    moving bounce-back with the wall velocity of the cell's
//                                  given values (getGivenRhoUxUyUz)
//   fluid cell, marker normal 1    forced-velocity cell: force rho (u_target - u) toward
//                                  the given velocity (the cases' getForcing hook,
//                                  M35Full/m35Main.cu:101-119)
//   every collided cell            plus the uniform body force, collided with the forcing
//                                  collision (M40Impeller/applyCollisionCustomized.h:6-16)
template <typename S>
__global__ void __launch_bounds__(kStepThreads) step_custom_kernel(const __grid_constant__ CustomParams<S> cp) {
  const StepParams<S>& p = cp.base;
  const uint32_t cell = blockIdx.x * kStepThreads + threadIdx.x;
  if (cell >= p.ri.n) return;
  const uint8_t m = p.marker[cell];
  const int kind = marker_kind(m);
  if (kind == kSkip) return;
  float f[27];
  load_cell_ri<S>(p.ri, cell, f);
  if (kind == kSolid) {
    if (marker_normal(m) == 1) {
      const float4 gv = p.given ? p.given[cell] : p.given_uniform;
      moving_bounceback(f, gv.y, gv.z, gv.w);
    } else {
#pragma unroll
      for (int q = 1; q < 27; q += 2) {
        const float t = f[q];
        f[q] = f[q + 1];
        f[q + 1] = t;
      }
    }
  } else {
    if (kind != kFluid) apply_boundary(m, f, p.given ? p.given[cell] : p.given_uniform);
    float gx = cp.body.x, gy = cp.body.y, gz = cp.body.z;
    if (kind == kFluid && marker_normal(m) == 1) {
      float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
      for (int q = 0; q < 27; ++q) {
        rho += f[q];
        jx += cx(q) * f[q];
        jy += cy(q) * f[q];
        jz += cz(q) * f[q];
      }
      const float4 gv = p.given ? p.given[cell] : p.given_uniform;
      gx += rho * (gv.y - jx / rho);
      gy += rho * (gv.z - jy / rho);
      gz += rho * (gv.w - jz / rho);
    }
    collide<true>(f, cell_relaxation(p.rx, p.cs, cell), gx, gy, gz);
    if (p.health) {
      const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
      if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
    }
  }
  store_cell_ri<S>(p.ri, cell, f);
}

// ------------------------------------------------------------------------------------------
// scalar transport (include/scalarTransportFunctions.h:10-176)
// ------------------------------------------------------------------------------------------
// Collision of the scalar populations T_q after the flow collision, after Zhang, Fan & Chen
// (2011, eqs 2.5-2.7) as applyScalarTransportCollision uses them: with the post-collision
// populations f, T_mean = sum f T / rho, S = sum c (f (T - T_mean)),
// F_q = 3/rho (c_q - u) . S and T_q <- T_mean + (1 - 1/tau_T) F_q.  sum f T is unchanged.
__device__ __forceinline__ void scalar_collision(const float (&f)[27], float (&T)[27], float tauT) {
  float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f, ft = 0.f;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    rho += f[q];
    jx += cx(q) * f[q];
    jy += cy(q) * f[q];
    jz += cz(q) * f[q];
    ft += f[q] * T[q];
  }
  const float inv_rho = 1.f / rho;
  const float ux = jx * inv_rho, uy = jy * inv_rho, uz = jz * inv_rho;
  const float tm = ft * inv_rho;
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    const float g = f[q] * (T[q] - tm);
    sx += cx(q) * g;
    sy += cy(q) * g;
    sz += cz(q) * g;
  }
  const float a = (1.f - 1.f / tauT) * 3.f * inv_rho;
#pragma unroll
  for (int q = 0; q < 27; ++q) T[q] = tm + a * ((cx(q) - ux) * sx + (cy(q) - uy) * sy + (cz(q) - uz) * sz);
}

template <typename S>
struct ScalarParams {
  StepParams<S> base;
  RowIndex<StoreF32> T;    // the scalar populations: FP32 rows at the flow rows' offsets
  const float* givenT;     // per-cell prescribed concentration (NaN: none), or null
  float tauT;
};

// applyLocalCellUpdate with scalar transport (scalarTransportFunctions.h:10-107): T is
// bounced back with f in solid cells, mirrored with f in free-slip cells, set to the given
// concentration where one is prescribed, and collided after the flow collision.
template <typename S>
__global__ void __launch_bounds__(kStepThreads) step_scalar_kernel(const __grid_constant__ ScalarParams<S> sp) {
  const StepParams<S>& p = sp.base;
  const uint32_t cell = blockIdx.x * kStepThreads + threadIdx.x;
  if (cell >= p.ri.n) return;
  const uint8_t m = p.marker[cell];
  const int kind = marker_kind(m);
  if (kind == kSkip) return;
  float f[27], T[27];
  load_cell_ri<S>(p.ri, cell, f);
  load_cell_ri<StoreF32>(sp.T, cell, T);
  if (kind == kSolid) {
#pragma unroll
    for (int q = 1; q < 27; q += 2) {
      const float a = f[q], b = T[q];
      f[q] = f[q + 1];
      f[q + 1] = a;
      T[q] = T[q + 1];
      T[q + 1] = b;
    }
  } else {
    if (kind != kFluid) {
      apply_boundary(m, f, p.given ? p.given[cell] : p.given_uniform);
      if (kind == kMirror) bc::mirror(marker_normal(m), T);
    }
    if (sp.givenT) {
      const float tg = sp.givenT[cell];
      if (tg == tg) {
#pragma unroll
        for (int q = 0; q < 27; ++q) T[q] = tg;
      }
    }
    collide<false>(f, cell_relaxation(p.rx, p.cs, cell));
    scalar_collision(f, T, sp.tauT);
    if (p.health) {
      const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
      if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
    }
  }
  store_cell_ri<S>(p.ri, cell, f);
  store_cell_ri<StoreF32>(sp.T, cell, T);
}

// Per-cell concentration sum f T / rho (FP64 sums) in logical order.
template <typename S>
__global__ void scalar_mean_kernel(GridView<S> g, GridView<StoreF32> t, double* out) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  double rho = 0.0, ft = 0.0;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    const uint32_t a = shifted(cell, g.shift[q], g.n);
    const double v = (double)S::load_q(g.fq[q] + a, q);
    rho += v;
    ft += v * (double)t.fq[q][a];
  }
  out[cell] = ft / rho;
}

// ------------------------------------------------------------------------------------------
// set-up kernels (hooks)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cell_ijk(uint32_t cell, const InfoStruct& I, int& i, int& j, int& k) {
  const uint32_t xy = (uint32_t)I.cellCountX * (uint32_t)I.cellCountY;
  k = (int)(cell / xy);
  const uint32_t r = cell - (uint32_t)k * xy;
  j = (int)(r / (uint32_t)I.cellCountX);
  i = (int)(r - (uint32_t)j * (uint32_t)I.cellCountX);
}

template <typename Case>
__global__ void fill_markers_kernel(Case c, InfoStruct I, uint32_t n, uint8_t* marker, float4* given) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= n) return;
  int i, j, k;
  cell_ijk(cell, I, i, j, k);
  MarkerStruct M;
  c.getMarkers(i, j, k, M, I);
  marker[cell] = encode_marker(i, j, k, M, I);
  if (given) {
    float rho = 1.f, ux = 0.f, uy = 0.f, uz = 0.f;
    c.getGivenRhoUxUyUz(i, j, k, rho, ux, uy, uz, I);
    given[cell] = make_float4(rho, ux, uy, uz);
  }
}

// second-order equilibrium (include/cellFunctions.h:60-121)
template <typename T>
__device__ __forceinline__ void equilibrium(T rho, T ux, T uy, T uz, T (&fe)[27]) {
  const T u2 = ux * ux + uy * uy + uz * uz;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    const T cu = (T)cx(q) * ux + (T)cy(q) * uy + (T)cz(q) * uz;
    fe[q] = rho * weight_t<T>(q) * (T(1) + T(3) * cu + T(4.5) * cu * cu - T(1.5) * u2);
  }
}

template <typename S, typename Case>
__global__ void fill_equilibrium_kernel(GridView<S> g, Case c, InfoStruct I) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  int i, j, k;
  cell_ijk(cell, I, i, j, k);
  MarkerStruct M;
  c.getMarkers(i, j, k, M, I);  // the start hook sees the cell's markers (fillEquilibrium.h:15-16)
  float rho = 1.f, ux = 0.f, uy = 0.f, uz = 0.f;
  c.getInitialRhoUxUyUz(i, j, k, rho, ux, uy, uz, M, I);
  using T = typename S::calc;
  T fe[27];
  equilibrium<T>(rho, ux, uy, uz, fe);
  store_cell<S>(g, cell, fe);
}

// fillEquilibrium with a field hook: rho_u holds four logical-order planes (rho, ux, uy, uz).
template <typename S>
__global__ void fill_equilibrium_field_kernel(GridView<S> g, const float* __restrict__ rho_u) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  const size_t n = g.n;
  using T = typename S::calc;
  T fe[27];
  equilibrium<T>(rho_u[cell], rho_u[n + cell], rho_u[2 * n + cell], rho_u[3 * n + cell], fe);
  store_cell<S>(g, cell, fe);
}

// ------------------------------------------------------------------------------------------
// periodic x / y fix-up after streaming (include/boundaryConditions/periodicXY.h:11-101):
// the 9 populations with c_x > 0 of the left face come from the right face, those with
// c_x < 0 of the right face from the left face (layers 0 and N-1 coincide).
// ------------------------------------------------------------------------------------------
template <typename S, int Axis>
__global__ void periodic_kernel(GridView<S> g, int nx, int ny, int nz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int na = Axis == 0 ? ny : nx;
  if (t >= na * nz) return;
  const int a = t % na, k = t / na;
  uint32_t left, right;
  if (Axis == 0) {
    left = ((uint32_t)k * ny + a) * nx;
    right = left + nx - 1;
  } else {
    left = ((uint32_t)k * ny) * nx + a;
    right = ((uint32_t)k * ny + (ny - 1)) * nx + a;
  }
#pragma unroll
  for (int q = 1; q < 27; ++q) {
    const int c = Axis == 0 ? cx(q) : cy(q);
    if (c > 0) {
      g.fq[q][shifted(left, g.shift[q], g.n)] = g.fq[q][shifted(right, g.shift[q], g.n)];
    } else if (c < 0) {
      g.fq[q][shifted(right, g.shift[q], g.n)] = g.fq[q][shifted(left, g.shift[q], g.n)];
    }
  }
}

// ------------------------------------------------------------------------------------------
// coarse <-> fine transfer (include/gridRefinementFunctions.h:283-526), two launches
//
// Phase 1 (restriction): every coarse cell on the surface of the box
//   [iS+1, iE-2] x [jS+1, jE-2] x [kS+1, kE-2] gets the average of its 8 fine children,
//   rescaled fine->coarse (writeToCoarseGridInterface; the reference's six face launches
//   overlap on edges and corners with identical values, here each cell is written once).
// Then, in a launch of its own:
// Phase 2 (prolongation): every fine cell in the two outer layers of each active face gets
//   the 7-point interpolation of the coarse field around its parent, rescaled
//   coarse->fine (writeToFineGridInterface).  Ghost cells receive only the populations of
//   the faces they belong to that stream inward (the union of those faces' 9-direction
//   sets); other cells receive all 27.  The reference runs six face launches in sequence;
//   since every launch computes the same value for a given fine cell, the union is the
//   same final state.
// ------------------------------------------------------------------------------------------
template <typename S>
struct CoarseFineParams {
  RowIndex<S> c;
  RowIndex<S> f;
  int cnx, cny, cnz;
  int iS, jS, kS, iE, jE, kE;
  int fnx, fny, fnz;
  const uint8_t* fine_marker;
  int face_active;          // bit 2*axis: start face, bit 2*axis+1: end face
  uint32_t n_ring;          // restriction work items
  uint32_t n_shell;         // prolongation work items
};

// direction sets streaming inward across each face (gridRefinementFunctions.h:441-446):
// dir_mask(axis, +1) for a start face, dir_mask(axis, -1) for an end face
constexpr uint32_t kAllDirs = (1u << 27) - 1;

// The prolongation's coarse reads use ordinary (L1-cached) loads: it is a launch of its own
// after the restriction's, and L1 starts empty for every launch, so no stale copy of a
// restricted ring cell can be hit.
// kFlat: the grid's rows are mapped twice (rows 2N apart), so cell + off_q needs no wrap.
template <bool kFlat = false, typename S>
__device__ __forceinline__ typename S::calc load_pop(const RowIndex<S>& r, int q, uint32_t cell) {
  if constexpr (kFlat) return S::load_q(r.base + (cell + r.off[q]), q);
  else return S::load_q(r.base + (cell + r.off[q] - (cell >= r.lim[q] ? r.n : 0u)), q);
}
template <bool kFlat = false, typename S>
__device__ __forceinline__ void store_pop(const RowIndex<S>& r, int q, uint32_t cell, typename S::calc v) {
  if constexpr (kFlat) S::store_q(r.base + (cell + r.off[q]), v, q);
  else S::store_q(r.base + (cell + r.off[q] - (cell >= r.lim[q] ? r.n : 0u)), v, q);
}

// Work items are dealt out in warp-sized chunks, consecutive chunks to consecutive blocks,
// so both phases spread over every SM while each warp still touches consecutive cells.
#define PSL_FOR_EACH_ITEM(t, count)                                                                        \
  for (uint32_t chunk_ = blockIdx.x + gridDim.x * (threadIdx.x >> 5); chunk_ * 32u < (count);            \
       chunk_ += gridDim.x * (blockDim.x >> 5))                                                            \
    for (uint32_t t = chunk_ * 32u + (threadIdx.x & 31u); t < (count); t = (count))

constexpr int kCoarseFineThreads = 128;

// Coarse cell (i, j, k) of the refined block from its 8 fine children: their populations
// added in the child order (k, j, i outer to inner), averaged, rescaled fine -> coarse
// (writeToCoarseGridInterface, gridRefinementFunctions.h:283-336).
template <bool kFlat = false, typename S>
__device__ __forceinline__ void restrict_cell(const RowIndex<S>& rc, const RowIndex<S>& rf, const CoarseFineParams<S>& p,
                                              int i, int j, int k) {
  using T = typename S::calc;
  const int fi = (i - p.iS) * 2, fj = (j - p.jS) * 2, fk = (k - p.kS) * 2;
  uint32_t fc[8];
#pragma unroll
  for (int c = 0; c < 8; ++c)
    fc[c] = ((uint32_t)(fk + (c >> 2)) * p.fny + (fj + ((c >> 1) & 1))) * p.fnx + (fi + (c & 1));
  // population by population (the eight children of one population are independent loads),
  // each summed in the child order
  T f[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    T v = T(0);
#pragma unroll
    for (int c = 0; c < 8; ++c) v = rn_add(v, load_pop<kFlat>(rf, q, fc[c]));
    f[q] = v * T(0.125);
  }
  rescale(f, false);
  const uint32_t cc = ((uint32_t)k * p.cny + j) * p.cnx + i;
#pragma unroll
  for (int q = 0; q < 27; ++q) store_pop<kFlat>(rc, q, cc, f[q]);
}

// fillCoarseGridFromFine (gridRefinementFunctions.h:528-535): every coarse cell of the box
// [iS+1, iE-1) x [jS+1, jE-1) x [kS+1, kE-1) -- the refined region inside the ring, ring
// included -- restricted from the fine grid (one thread per coarse cell, i fastest).
template <typename S>
__global__ void __launch_bounds__(kCoarseFineThreads) fill_coarse_kernel(const __grid_constant__ CoarseFineParams<S> p) {
  const uint32_t a = p.iE - p.iS - 2, b = p.jE - p.jS - 2, c = p.kE - p.kS - 2;
  const uint32_t t = blockIdx.x * kCoarseFineThreads + threadIdx.x;
  if (t >= a * b * c) return;
  restrict_cell(p.c, p.f, p, p.iS + 1 + (int)(t % a), p.jS + 1 + (int)((t / a) % b), p.kS + 1 + (int)(t / (a * b)));
}

// kPhase 1: the restriction, 2: the prolongation, as two ordinary launches in stream order
// (the launch boundary orders them; one cooperative launch with a grid barrier between the
// phases ran 0.174 / 0.167 ms per FP32 / FP16 transfer against 0.168 / 0.154 for the two).
// kFlat: both grids' rows are mapped twice (no wrap test on any population address).
template <typename S, int kPhase, bool kFlat>
__global__ void __launch_bounds__(kCoarseFineThreads) coarse_fine_kernel(const __grid_constant__ CoarseFineParams<S> p) {
  using T = typename S::calc;
  // The row offsets of both grids are read from shared memory inside the item loops (kept
  // as kernel parameters, the compiler holds all of them in registers across iterations).
  __shared__ RowIndex<S> rc, rf;
  if (threadIdx.x < 27) {
    rc.off[threadIdx.x] = p.c.off[threadIdx.x];
    rc.lim[threadIdx.x] = p.c.lim[threadIdx.x];
    rf.off[threadIdx.x] = p.f.off[threadIdx.x];
    rf.lim[threadIdx.x] = p.f.lim[threadIdx.x];
  }
  if (threadIdx.x == 0) {
    rc.base = p.c.base;
    rc.n = p.c.n;
    rf.base = p.f.base;
    rf.n = p.f.n;
  }
  __syncthreads();
  // ---------------- phase 1: restriction ----------------
  if (kPhase != 2) {
    const int a = p.iE - p.iS - 2, b = p.jE - p.jS - 2, c = p.kE - p.kS - 2;  // ring box extents
    const uint32_t faceK = 2u * a * b;
    const uint32_t faceJ = 2u * a * (c - 2);
    PSL_FOR_EACH_ITEM(t, p.n_ring) {
      int ri, rj, rk;
      if (t < faceK) {
        const uint32_t layer = t / (a * b), r = t % (a * b);
        rk = layer ? c - 1 : 0;
        rj = r / a;
        ri = r % a;
      } else if (t < faceK + faceJ) {
        const uint32_t u = t - faceK, layer = u / (a * (c - 2)), r = u % (a * (c - 2));
        rj = layer ? b - 1 : 0;
        rk = 1 + r / a;
        ri = r % a;
      } else {
        // x faces: neighbouring lanes take the start- and end-face ring cells of one (j, k), so
        // a warp reads both ends of the same fine rows, whose child pairs share sectors
        const uint32_t u = t - faceK - faceJ, r = u >> 1;
        ri = (u & 1u) ? a - 1 : 0;
        rj = 1 + r % (b - 2);
        rk = 1 + r / (b - 2);
      }
      restrict_cell<kFlat>(rc, rf, p, p.iS + 1 + ri, p.jS + 1 + rj, p.kS + 1 + rk);
    }
  }
  if (kPhase == 1) return;
  // ---------------- phase 2: prolongation ----------------
  const uint32_t kPos[3] = {dir_mask(0, 1), dir_mask(1, 1), dir_mask(2, 1)};
  const uint32_t kNeg[3] = {dir_mask(0, -1), dir_mask(1, -1), dir_mask(2, -1)};
  const int nx = p.fnx, ny = p.fny, nz = p.fnz;
  const uint32_t zl = 4u * nx * ny, yl = 4u * nx * (nz - 4);
  PSL_FOR_EACH_ITEM(t, p.n_shell) {
    int i, j, k;
    if (t < zl) {
      const uint32_t layer = t / (nx * ny), r = t % (nx * ny);
      k = layer < 2 ? layer : nz - 4 + layer;
      j = r / nx;
      i = r % nx;
    } else if (t < zl + yl) {
      const uint32_t u = t - zl, layer = u / (nx * (nz - 4)), r = u % (nx * (nz - 4));
      j = layer < 2 ? layer : ny - 4 + layer;
      k = 2 + r / nx;
      i = r % nx;
    } else {
      // x faces: four lanes per row boundary take the end of row j - 1 (i = Nx - 2, Nx - 1)
      // and the start of row j (i = 0, 1), four consecutive cells in memory, so each
      // population's store covers 16 contiguous bytes; at j = 2 and j = Ny - 2 one side of
      // the boundary is a y-face row (its cells are y-face items) and those lanes idle
      const uint32_t u = t - zl - yl, per_k = 4u * (ny - 3);
      const uint32_t b = (u % per_k) >> 2, sub = u & 3u;
      k = 2 + (int)(u / per_k);
      j = 2 + (int)b - (sub < 2 ? 1 : 0);
      i = sub < 2 ? nx - 2 + (int)sub : (int)sub - 2;
      if (j < 2 || j >= ny - 2) continue;
    }
    const uint32_t fcell = ((uint32_t)k * ny + j) * nx + i;
    const uint8_t fm = p.fine_marker[fcell];
    const bool ghost = marker_kind(fm) == kSkip && marker_normal(fm) == 1;
    const int idx[3] = {i, j, k};
    const int dim[3] = {nx, ny, nz};
    uint32_t mask = 0;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      if ((p.face_active >> (2 * ax)) & 1)
        if (idx[ax] < 2) mask |= ghost ? kPos[ax] : kAllDirs;
      if ((p.face_active >> (2 * ax + 1)) & 1)
        if (idx[ax] >= dim[ax] - 2) mask |= ghost ? kNeg[ax] : kAllDirs;
    }
    if (!mask) continue;
    const int ic = i / 2 + p.iS, jc = j / 2 + p.jS, kc = k / 2 + p.kS;
    const T d[3] = {T((i & 1) ? 0.25f : -0.25f), T((j & 1) ? 0.25f : -0.25f), T((k & 1) ? 0.25f : -0.25f)};
    const uint32_t pc = ((uint32_t)kc * p.cny + jc) * p.cnx + ic;
    const int cidx[3] = {ic, jc, kc};
    const int cdim[3] = {p.cnx, p.cny, p.cnz};
    uint32_t nc[6];  // the six neighbours in the order (x+, x-, y+, y-, z+, z-)
    T w[6];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      int plus = cidx[ax] + 1, minus = cidx[ax] - 1;
      T inv = T(0.5);
      if (plus >= cdim[ax]) { plus = cidx[ax]; inv = T(1); }
      if (minus < 0) { minus = 0; inv = T(1); }
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        int nb[3] = {ic, jc, kc};
        nb[ax] = side == 0 ? plus : minus;
        w[2 * ax + side] = (side == 0 ? inv : -inv) * d[ax];  // exact: powers of two
        nc[2 * ax + side] = ((uint32_t)nb[2] * p.cny + nb[1]) * p.cnx + nb[0];
      }
    }
    // population by population, the parent first and then the six neighbours in that order
    T f[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      T v = load_pop<kFlat>(rc, q, pc);
#pragma unroll
      for (int t = 0; t < 6; ++t) v = rn_add(v, load_pop<kFlat>(rc, q, nc[t]) * w[t]);
      f[q] = v;
    }
    rescale(f, true);
#pragma unroll
    for (int q = 0; q < 27; ++q)
      if (mask & (1u << q)) store_pop<kFlat>(rf, q, fcell, f[q]);
  }
}

// ------------------------------------------------------------------------------------------
// momentum-exchange force on the solid cells of a box, FP64
// (getSphereDrag, flowAroundSphereMainSingle.cu:99-156; per cell rho*(u - u_bounced))
// Deterministic: per-block partial sums, then one block sums them in block order.
// ------------------------------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(256) force_partial_kernel(GridView<S> g, const uint8_t* marker, int nx, int ny,
                                                            int i0, int j0, int k0, int si, int sj, int sk,
                                                            double* partial) {
  const uint32_t total = (uint32_t)si * sj * sk;
  double acc[3] = {0.0, 0.0, 0.0};
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int i = i0 + (int)(t % si), j = j0 + (int)((t / si) % sj), k = k0 + (int)(t / (si * sj));
    const uint32_t cell = ((uint32_t)k * ny + j) * nx + i;
    if (marker_kind(marker[cell]) != kSolid) continue;
    double rho = 0, jx = 0, jy = 0, jz = 0, bx = 0, by = 0, bz = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      const double v = (double)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
      rho += v;
      jx += cx(q) * v;
      jy += cy(q) * v;
      jz += cz(q) * v;
      // the bounced population of direction q sits in direction opposite(q)
      bx -= cx(q) * v;
      by -= cy(q) * v;
      bz -= cz(q) * v;
    }
    acc[0] += rho * (jx / rho - bx / rho);
    acc[1] += rho * (jy / rho - by / rho);
    acc[2] += rho * (jz / rho - bz / rho);
  }
  __shared__ double red[3][256];
  for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int c = 0; c < 3; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < 3; ++c) partial[blockIdx.x * 3 + c] = red[c][0];
}

// The partial sums added in block order by one thread (deterministic); every thread of the
// block first stages a chunk of them in shared memory, so the serial sum waits on shared
// memory instead of one global load after another.  One block, any number of threads.
static __global__ void force_final_kernel(const double* partial, int nblocks, double* out) {
  constexpr int kChunk = 512;  // blocks per staged chunk (12 KB)
  __shared__ double stage[kChunk * 3];
  double s[3] = {0, 0, 0};
  for (int b0 = 0; b0 < nblocks; b0 += kChunk) {
    const int nb = min(kChunk, nblocks - b0);
    for (int i = threadIdx.x; i < nb * 3; i += blockDim.x) stage[i] = partial[b0 * 3 + i];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int b = 0; b < nb; ++b)
        for (int c = 0; c < 3; ++c) s[c] += stage[b * 3 + c];
    __syncthreads();
  }
  if (threadIdx.x == 0 && blockIdx.x == 0)
    for (int c = 0; c < 3; ++c) out[c] = s[c];
}

// ------------------------------------------------------------------------------------------
// logical-order gather / scatter (host I/O; population q of cell c at [q][c])
// ------------------------------------------------------------------------------------------
template <typename S>
__global__ void gather_logical_kernel(GridView<S> g, int q, float* out) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  out[cell] = S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
}
template <typename S>
__global__ void scatter_logical_kernel(GridView<S> g, int q, const float* in) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  S::store_q(g.fq[q] + shifted(cell, g.shift[q], g.n), in[cell], q);
}

// Density and velocity of every cell in FP64 (getRhoUxUyUz, cellFunctions.h:135-155),
// written as four logical-order planes.
template <typename S>
__global__ void macroscopic_kernel(GridView<S> g, double* out) {
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= g.n) return;
  double rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    const double v = (double)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
    rho += v;
    jx += cx(q) * v;
    jy += cy(q) * v;
    jz += cz(q) * v;
  }
  const size_t n = g.n;
  out[cell] = rho;
  out[n + cell] = jx / rho;
  out[2 * n + cell] = jy / rho;
  out[3 * n + cell] = jz / rho;
}

// ------------------------------------------------------------------------------------------
// single-cell entry points (unit-level parity of the device functions)
// ------------------------------------------------------------------------------------------
static __global__ void debug_cell_kernel(int op, int a0, float* f, const float* args, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  float v[27];
  float* base = f + (size_t)t * 27;
  for (int q = 0; q < 27; ++q) v[q] = base[q];
  const float* a = args + (size_t)t * 4;
  switch (op) {
    case 0: {  // collision (a: nu, cs)
      Relaxation rx;
      rx.tau = 3.f * a[0] + 0.5f;
      rx.tau2 = rx.tau * rx.tau;
      rx.omega0 = 1.f / rx.tau;
      rx.cs18 = 18.f * a[1];
      collide<false>(v, rx);
      break;
    }
    case 1: rescale(v, a0 != 0); break;
    case 2: bc::mbbc(a0, v, a[0], a[1], a[2], a[3]); break;
    case 3: {
      float rho = a[0], ux = a[1], uy = a[2], uz = a[3];
      bc::restore_rho(a0, v, rho, ux, uy, uz);
      v[0] = rho;
      break;
    }
    case 4: {
      float rho = a[0], ux = a[1], uy = a[2], uz = a[3];
      bc::restore_u(a0, v, rho, ux, uy, uz);
      v[0] = ux; v[1] = uy; v[2] = uz;
      break;
    }
    case 5: {
      float rho = a[0], ux = a[1], uy = a[2], uz = a[3];
      bc::restore_rho_u(a0, v, rho, ux, uy, uz);
      v[0] = rho; v[1] = ux; v[2] = uy; v[3] = uz;
      break;
    }
    case 6: bc::mirror(a0, v); break;
    case 7: {  // forced collision (a: nu, cs, gx; gy=gz=a[3])
      Relaxation rx;
      rx.tau = 3.f * a[0] + 0.5f;
      rx.tau2 = rx.tau * rx.tau;
      rx.omega0 = 1.f / rx.tau;
      rx.cs18 = 18.f * a[1];
      collide<true>(v, rx, a[2], a[3], 0.f);
      break;
    }
    default: break;
  }
  for (int q = 0; q < 27; ++q) base[q] = v[q];
}

}  // namespace psl
