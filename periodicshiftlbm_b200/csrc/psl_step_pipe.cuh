// The per-cell update as a pipeline of bulk copies (TMA, sm_100a): each CTA walks tiles
// of 128 consecutive cells (tile b, b + G, b + 2G, ... for CTA b of G resident CTAs).
// While its threads collide one tile out of shared memory, the copy engine is already
// bringing the next tiles in, so the bytes in flight no longer depend on how many warps
// are waiting on their own loads, and the populations' loads, stores and address
// arithmetic leave the instruction stream.
//
// Tile of cells [c0, c0 + L).  For population q its elements are the run [a, a + L) of
// row q, a = (c0 + shift_q) mod N (getShiftedIndex, include/applyStreaming.h:33-41),
// wrapping past N at most once.  Warp 0 lane q copies the run's 16-byte-aligned cover
// [a0, ...) into shared row q (one bulk copy, two when the run wraps; N is a multiple of
// 16 bytes, so the wrap point is aligned too), lane 27 the tile's marker bytes and lane 28
// its per-cell Smagorinsky constants when the grid has them; all count on the stage's
// mbarrier.  Cell c0 + t finds population q at shared element rem_q + t with
// rem_q = shift_q mod (16 / element size), the same for every tile of a launch.
//
// After the update (in place in shared memory, each thread its own cell), lane q writes
// its run back: the aligned interior as one bulk store, the ragged ends (< 16 bytes each)
// as at most three aligned plain stores each.  Those end chunks also hold elements that
// belong to the neighbouring tiles' cells, which are read here but never written, so every
// (population, address) pair is still written only by its own cell and the in-place PS
// update stays race-free (include/applyLocalCellUpdate.h:34,71).
//
// Stages: kStages buffers of one tile each, loads issued kAhead tiles ahead.  A stage is
// refilled only after the bulk stores that read it have finished reading
// (cp.async.bulk.wait_group.read); every mbarrier wait is bounded, and a wait that runs
// out sets health bit 2 and ends the CTA after letting its copies in flight land.
//
// Arithmetic per cell: FP32 storage runs collide<false> (psl_collision.cuh, the
// reference's operation order, bit for bit the one-thread-per-cell kernel's result);
// FP16 / BF16 storage collides the stored deviations g = f - w directly
// (psl_collision_g.cuh).
#pragma once
#include "psl_async.cuh"
#include "psl_collision_g.cuh"
#include "psl_kernels.cuh"

namespace psl {

constexpr int kPipeCells = 128;            // cells per tile = threads per CTA
constexpr uint32_t kPipePolls = 1u << 22;  // bounded mbarrier waits

template <typename S>
struct PipeTraits;
template <>
struct PipeTraits<StoreF32> {
  static constexpr int kStages = 3, kAhead = 1;
};
template <>
struct PipeTraits<StoreF16> {
  static constexpr int kStages = 4, kAhead = 2;
};
template <>
struct PipeTraits<StoreBF16> {
  static constexpr int kStages = 4, kAhead = 2;
};

template <typename S>
struct PipeLayout {
  using T = typename S::type;
  static constexpr int E = sizeof(T);
  static constexpr int V = 16 / E;                          // elements per 16-byte chunk
  static constexpr int R = kPipeCells + V;                  // shared row length (aligned cover)
  static constexpr int kRowBytes = R * E;                   // multiple of 16
  static constexpr int kMarkerOff = 27 * kRowBytes;         // 128 marker bytes
  static constexpr int kCsOff = kMarkerOff + kPipeCells;    // 128 FP32 C_s (when present)
  static constexpr int kStageBytes = kCsOff;                // without the C_s field
  static constexpr int kStageBytesCs = kCsOff + 4 * kPipeCells;
  static constexpr int kStages = PipeTraits<S>::kStages;
  static constexpr int kAhead = PipeTraits<S>::kAhead;
  static_assert(kAhead >= 1 && kAhead < kStages, "look-ahead must leave a stage to compute in");
  static_assert(kRowBytes % 16 == 0 && kMarkerOff % 16 == 0 && kCsOff % 16 == 0, "16-byte aligned regions");
};

template <typename S>
struct PipeParams {
  typename S::type* base;  // population row q at base + q * stride
  uint32_t stride;         // elements per row (multiple of 64)
  uint32_t n;              // cells, a multiple of 16 / sizeof(element)
  uint32_t ntiles;
  uint32_t stage_bytes;    // PipeLayout kStageBytes, or kStageBytesCs with a C_s field
  uint32_t extra_bytes;    // 16 bytes for every row whose runs start unaligned
  uint32_t shift[27];
  uint32_t soff[27];       // byte offset of tile cell 0's element in a stage: q * kRowBytes + rem_q * E
  const uint8_t* marker;
  const float4* given;     // per-cell (rho, ux, uy, uz) of boundary cells, or null
  float4 given_uniform;
  const float* cs;         // per-cell Smagorinsky constant, or null: rx.cs18 everywhere
  RelaxationT<float> rx;
  unsigned int* health;
};

template <typename S>
__device__ __forceinline__ float raw_to_float(const void* p);
template <>
__device__ __forceinline__ float raw_to_float<StoreF32>(const void* p) { return *static_cast<const float*>(p); }
template <>
__device__ __forceinline__ float raw_to_float<StoreF16>(const void* p) { return __half2float(*static_cast<const __half*>(p)); }
template <>
__device__ __forceinline__ float raw_to_float<StoreBF16>(const void* p) {
  return __bfloat162float(*static_cast<const __nv_bfloat16*>(p));
}
template <typename S>
__device__ __forceinline__ void float_to_raw(void* p, float v);
template <>
__device__ __forceinline__ void float_to_raw<StoreF32>(void* p, float v) { *static_cast<float*>(p) = v; }
template <>
__device__ __forceinline__ void float_to_raw<StoreF16>(void* p, float v) { *static_cast<__half*>(p) = __float2half_rn(v); }
template <>
__device__ __forceinline__ void float_to_raw<StoreBF16>(void* p, float v) {
  *static_cast<__nv_bfloat16*>(p) = __float2bfloat16_rn(v);
}

// Warp 0: bulk loads of tile [c0, c0 + L) into a stage, counted on its mbarrier.
template <typename S>
__device__ __forceinline__ void pipe_issue_loads(const PipeParams<S>& p, uint32_t c0, unsigned char* st, uint64_t* bar,
                                                 int lane) {
  using Lay = PipeLayout<S>;
  constexpr uint32_t V = Lay::V, E = Lay::E;
  const uint32_t L = min((uint32_t)kPipeCells, p.n - c0);
  if (lane == 0)
    mbar_arrive_expect_tx(bar, 27u * L * E + p.extra_bytes + ((L + 15u) & ~15u) + (p.cs ? 4u * L : 0u));
  __syncwarp();
  if (lane < 27) {
    uint32_t a = c0 + p.shift[lane];
    if (a >= p.n) a -= p.n;
    const uint32_t a0 = a & ~(V - 1);
    const typename S::type* row = p.base + (size_t)lane * p.stride;
    unsigned char* dst = st + lane * Lay::kRowBytes;
    if (a + L <= p.n) {
      bulk_load(dst, row + a0, (((a + L + V - 1) & ~(V - 1)) - a0) * E, bar);
    } else {
      bulk_load(dst, row + a0, (p.n - a0) * E, bar);
      bulk_load(dst + (p.n - a0) * E, row, ((a + L - p.n + V - 1) & ~(V - 1)) * E, bar);
    }
  } else if (lane == 27) {
    bulk_load(st + Lay::kMarkerOff, p.marker + c0, (L + 15u) & ~15u, bar);
  } else if (lane == 28 && p.cs) {
    bulk_load(st + Lay::kCsOff, p.cs + c0, 4u * L, bar);
  }
}

// Copies k elements (k * E = 2, 4 or 8 bytes, aligned) from shared to global memory.
template <int Bytes>
__device__ __forceinline__ void copy_piece(unsigned char* g, const unsigned char* s) {
  if constexpr (Bytes == 2) *reinterpret_cast<uint16_t*>(g) = *reinterpret_cast<const uint16_t*>(s);
  if constexpr (Bytes == 4) *reinterpret_cast<uint32_t*>(g) = *reinterpret_cast<const uint32_t*>(s);
  if constexpr (Bytes == 8) *reinterpret_cast<uint2*>(g) = *reinterpret_cast<const uint2*>(s);
}

// Elements [g0, g1) of a global row from shared memory, element x at byte (x - x0) * E of
// `srow` (x0: the 16-byte-aligned global element the shared row starts with, so shared
// and global addresses agree modulo 16; x - x0 is taken modulo 2^32, which is how the
// wrapped part of a run finds its place after the part before the wrap point): the
// aligned interior as one bulk store, each ragged end as at most three aligned stores.
template <typename S>
__device__ __forceinline__ void pipe_write_segment(typename S::type* row, const unsigned char* srow, uint32_t x0,
                                                   uint32_t g0, uint32_t g1) {
  using Lay = PipeLayout<S>;
  constexpr uint32_t V = Lay::V, E = Lay::E;
  unsigned char* grow = reinterpret_cast<unsigned char*>(row);
  auto gp = [&](uint32_t x) { return grow + (size_t)x * E; };
  auto sp = [&](uint32_t x) { return srow + (x - x0) * E; };
  const uint32_t h0 = (g0 + V - 1) & ~(V - 1), h1 = g1 & ~(V - 1);
  if (h1 <= h0) {  // no aligned interior: a short piece next to the wrap point
    for (uint32_t x = g0; x < g1; ++x) copy_piece<E>(gp(x), sp(x));
    return;
  }
  uint32_t x = g0;  // head: align x up to V elements with pieces of 1, 2, 4 elements
  if (E == 2 && (x & 1u)) {
    copy_piece<2>(gp(x), sp(x));
    x += 1;
  }
  if (x & (4u / E)) {
    copy_piece<4>(gp(x), sp(x));
    x += 4u / E;
  }
  if (x & (8u / E)) {
    copy_piece<8>(gp(x), sp(x));
    x += 8u / E;
  }
  bulk_store(gp(h0), sp(h0), (h1 - h0) * E);
  x = h1;  // tail: g1 - h1 < V elements
  const uint32_t r = g1 - h1;
  if (r & (8u / E)) {
    copy_piece<8>(gp(x), sp(x));
    x += 8u / E;
  }
  if (r & (4u / E)) {
    copy_piece<4>(gp(x), sp(x));
    x += 4u / E;
  }
  if (E == 2 && (r & 1u)) copy_piece<2>(gp(x), sp(x));
}

// Warp 0: write tile [c0, c0 + L) back from its stage, then commit the lane's bulk group.
template <typename S>
__device__ __forceinline__ void pipe_store_tile(const PipeParams<S>& p, const unsigned char* st, uint32_t c0,
                                                int lane) {
  using Lay = PipeLayout<S>;
  constexpr uint32_t V = Lay::V;
  if (lane < 27) {
    const uint32_t L = min((uint32_t)kPipeCells, p.n - c0);
    uint32_t a = c0 + p.shift[lane];
    if (a >= p.n) a -= p.n;
    const uint32_t a0 = a & ~(V - 1);
    typename S::type* row = p.base + (size_t)lane * p.stride;
    const unsigned char* srow = st + lane * Lay::kRowBytes;
    if (a + L <= p.n) {
      pipe_write_segment<S>(row, srow, a0, a, a + L);
    } else {
      pipe_write_segment<S>(row, srow, a0, a, p.n);
      pipe_write_segment<S>(row, srow, a0 - p.n, 0, a + L - p.n);  // x - (a0 - N) = x + N - a0
    }
  }
  bulk_commit();
}

// One cell of a tile, in place in the stage (applyLocalCellUpdate.h:21-72).
template <typename S>
__device__ __forceinline__ void pipe_update_cell(const PipeParams<S>& p, unsigned char* st, int t, uint32_t cell,
                                                 float* slot) {
  using Lay = PipeLayout<S>;
  using T = typename S::type;
  const uint8_t m = st[Lay::kMarkerOff + t];
  const int kind = marker_kind(m);
  if (kind == kSkip) return;
  unsigned char* mine = st + t * Lay::E;
  if (kind == kSolid) {  // bounce-back: g and f swap alike (w_q = w_opposite(q))
#pragma unroll
    for (int q = 1; q < 27; q += 2) {
      T* a = reinterpret_cast<T*>(mine + p.soff[q]);
      T* b = reinterpret_cast<T*>(mine + p.soff[q + 1]);
      const T x = *a;
      *a = *b;
      *b = x;
    }
    return;
  }
  float v[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) v[q] = raw_to_float<S>(mine + p.soff[q]);
  const float cs18 = p.cs ? 18.f * *reinterpret_cast<const float*>(st + Lay::kCsOff + 4 * t) : p.rx.cs18;
  if constexpr (S::kind == kStoreF32) {
    if (kind != kFluid) apply_boundary_at(m, v, p.given ? p.given[cell] : p.given_uniform, slot);
    RelaxationT<float> rx = p.rx;
    rx.cs18 = cs18;
    collide<false>(v, rx);
    if (p.health) {
      const float r = v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6];
      if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
    }
  } else {
    if (kind != kFluid) {  // the boundary functions work on f
#pragma unroll
      for (int q = 0; q < 27; ++q) v[q] += lattice_weight(q);
      apply_boundary_at(m, v, p.given ? p.given[cell] : p.given_uniform, slot);
#pragma unroll
      for (int q = 0; q < 27; ++q) v[q] -= lattice_weight(q);
    }
    const CellMomentsG cm = cell_moments_g(v);
    if (p.health && !(cm.rho > 0.f && cm.rho < 1.0e30f)) atomicOr(p.health, 1u);
    relax_rebuild_g(v, cm, smagorinsky_omega_g(cm, p.rx.omega0, p.rx.tau, p.rx.tau2, cs18));
  }
#pragma unroll
  for (int q = 0; q < 27; ++q) float_to_raw<S>(mine + p.soff[q], v[q]);
}

// The pipeline around a per-cell body: body(st, t, cell, active) runs on every thread of
// the CTA for each of its tiles (st: the tile's stage, active: cell c0 + t exists), so a
// body may use warp-wide operations.
template <typename S, typename Body>
__device__ __forceinline__ void pipe_run(const PipeParams<S>& p, unsigned char* smem, Body&& body) {
  using Lay = PipeLayout<S>;
  constexpr int kS = Lay::kStages, kD = Lay::kAhead;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kS * p.stage_bytes);
  const int t = threadIdx.x, lane = t & 31;
  const bool producer = t < 32;
  if (t == 0) {
#pragma unroll
    for (int s = 0; s < kS; ++s) mbar_init(&full[s], 1);
    mbar_init_fence();
  }
  __syncthreads();
  const uint32_t G = gridDim.x, b = blockIdx.x;
  const uint32_t count = b < p.ntiles ? (p.ntiles - 1 - b) / G + 1 : 0;
  if (producer)
    for (uint32_t d = 0; d < (uint32_t)kD && d < count; ++d)
      pipe_issue_loads(p, (b + d * G) * kPipeCells, smem + d * p.stage_bytes, &full[d], lane);
  for (uint32_t j = 0; j < count; ++j) {
    if (producer && j + kD < count) {
      const uint32_t s2 = (j + kD) % kS;
      bulk_wait_read<kS - kD - 1>();  // the stores that last read stage s2 are done reading
      fence_proxy_async_smem();
      pipe_issue_loads(p, (b + (j + kD) * G) * kPipeCells, smem + s2 * p.stage_bytes, &full[s2], lane);
    }
    const uint32_t s = j % kS;
    unsigned char* st = smem + s * p.stage_bytes;
    const uint32_t c0 = (b + j * G) * kPipeCells;
    // warp-uniform, so a body's warp-wide steps run on all of a warp's lanes or on none
    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&full[s], (j / kS) & 1u, kPipePolls));
    if (ok) body(st, t, c0 + t, c0 + t < p.n);
    fence_proxy_async_smem();
    if (!__syncthreads_and(ok)) {
      // a tile did not arrive in time: flag it, let every load still in flight land
      // (bounded as well), and end this CTA
      if (t == 0 && p.health) atomicOr(p.health, 4u);
      if (t == 0)
        for (uint32_t jj = j; jj < count && jj <= j + kD; ++jj)
          mbar_wait_bounded(&full[jj % kS], (jj / kS) & 1u, kPipePolls);
      break;
    }
    if (producer) pipe_store_tile<S>(p, st, c0, lane);
  }
  if (producer) bulk_wait_all();
}

template <typename S>
__global__ void __launch_bounds__(kPipeCells) step_pipe_kernel(const __grid_constant__ PipeParams<S> p) {
  __shared__ __align__(16) float bc_slot[kPipeCells][27];
  extern __shared__ __align__(128) unsigned char smem[];
  pipe_run<S>(p, smem, [&](unsigned char* st, int t, uint32_t cell, bool active) {
    if (active) pipe_update_cell<S>(p, st, t, cell, bc_slot[t]);
  });
}

}  // namespace psl
