// Tiled per-cell update: the population rows of a 128-cell block move between HBM and
// shared memory as TMA bulk copies; threads collide from and to shared memory.
//
// For population q the block's 128 cells own the consecutive addresses
// [a, a + 128) with a = shifted(c0, shift_q) (wrapping once past N at most).  Warp 0 lanes
// 0..26 each copy their row's 16-byte-aligned cover [a0, a1) of that run into shared
// memory (one bulk copy, two when it wraps), counted on one mbarrier.  After the update,
// the same lanes write back the aligned interior of the run with bulk stores and the at
// most V-1 elements at each ragged end with plain stores: those boundary 16-byte chunks
// also hold elements owned by neighbouring blocks, which are read here but never written.
// Each (population, address) pair is still written only by its owning cell, so the
// in-place update stays race-free (applyLocalCellUpdate.h:34,71).
//
// Requirements (checked by the host): N % 128 == 0 (so every block is full and the wrap
// point N is 16-byte aligned), rows 16-byte aligned.  A block whose cells are all skipped
// (refined interior, ghost layer) moves no data at all.
#pragma once
#include "psl_async.cuh"
#include "psl_kernels.cuh"

namespace psl {

constexpr int kTile = 128;                 // cells (= threads) per block
constexpr uint32_t kMaxMbarPolls = 1u << 22;  // bounded wait for the bulk loads

template <typename S>
struct TileRows {
  using T = typename S::type;
  static constexpr int E = sizeof(T);
  static constexpr int V = 16 / E;         // elements per 16-byte chunk
  static constexpr int R = kTile + 2 * V;  // shared row length (cover of an unaligned run)
  alignas(128) T rows[27][R];
  uint64_t bar;
  int off[27];                             // index of cell c0's element in shared row q
};

template <typename S, int Q = 0>
__device__ __forceinline__ void load_tile(const TileRows<S>& sh, int t, float (&f)[27]) {
  if constexpr (Q < 27) {
    f[Q] = S::template load<Q>(&sh.rows[Q][sh.off[Q] + t]);
    load_tile<S, Q + 1>(sh, t, f);
  }
}
template <typename S, int Q = 0>
__device__ __forceinline__ void store_tile(TileRows<S>& sh, int t, const float (&f)[27]) {
  if constexpr (Q < 27) {
    S::template store<Q>(&sh.rows[Q][sh.off[Q] + t], f[Q]);
    store_tile<S, Q + 1>(sh, t, f);
  }
}

// Write one global segment [g0, g1) of row q from shared row index s: bulk store of the
// aligned interior, plain stores for the ragged ends.
template <typename S>
__device__ __forceinline__ void write_segment(typename S::type* row, const typename S::type* srow, uint32_t g0,
                                              uint32_t g1, uint32_t s) {
  constexpr uint32_t V = TileRows<S>::V;
  constexpr uint32_t E = TileRows<S>::E;
  const uint32_t h0 = (g0 + V - 1) & ~(V - 1);
  const uint32_t h1 = g1 & ~(V - 1);
  if (h1 <= h0) {
    for (uint32_t x = g0; x < g1; ++x) row[x] = srow[s + (x - g0)];
    return;
  }
  for (uint32_t x = g0; x < h0; ++x) row[x] = srow[s + (x - g0)];
  bulk_store(row + h0, srow + s + (h0 - g0), (h1 - h0) * E);
  for (uint32_t x = h1; x < g1; ++x) row[x] = srow[s + (x - g0)];
}

template <typename S>
__global__ void __launch_bounds__(kTile) step_tiled_kernel(const __grid_constant__ StepParams<S> p) {
  using T = typename S::type;
  constexpr uint32_t V = TileRows<S>::V;
  constexpr uint32_t E = TileRows<S>::E;
  __shared__ TileRows<S> sh;
  const uint32_t n = p.g.n;
  const uint32_t c0 = blockIdx.x * kTile;
  const int t = threadIdx.x;
  const uint8_t m = p.marker[c0 + t];
  const int kind = marker_kind(m);
  if (t == 0) {
    mbar_init(&sh.bar, 1);
    mbar_init_fence();
  }
  if (!__syncthreads_or(kind != kSkip)) return;  // nothing to update: no data moves

  // ---- warp 0: bulk-load the 27 row runs ----
  if (t < 32) {
    const T* src1 = nullptr;
    const T* src2 = nullptr;
    uint32_t b1 = 0, b2 = 0, dst2 = 0;
    if (t < 27) {
      const uint32_t a = shifted(c0, p.g.shift[t], n);
      const uint32_t a0 = a & ~(V - 1);
      sh.off[t] = (int)(a - a0);
      src1 = p.g.fq[t] + a0;
      if (a + kTile <= n) {
        b1 = (((a + kTile + V - 1) & ~(V - 1)) - a0) * E;  // <= N: N is a multiple of V
      } else {
        b1 = (n - a0) * E;  // up to the wrap point, then from element 0
        src2 = p.g.fq[t];
        b2 = ((a + kTile - n + V - 1) & ~(V - 1)) * E;
        dst2 = n - a0;
      }
    }
    uint32_t bytes = b1 + b2;
#pragma unroll
    for (int o = 16; o; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    if (t == 0) mbar_arrive_expect_tx(&sh.bar, bytes);
    __syncwarp();
    if (t < 27) {
      bulk_load(&sh.rows[t][0], src1, b1, &sh.bar);
      if (b2) bulk_load(&sh.rows[t][dst2], src2, b2, &sh.bar);
    }
  }
  __syncthreads();  // off[] written
  if (!mbar_wait_bounded(&sh.bar, 0, kMaxMbarPolls)) {
    if (t == 0 && p.health) atomicOr(p.health, 4u);
    mbar_wait_bounded(&sh.bar, 0, kMaxMbarPolls);  // let copies in flight land before exiting
    return;
  }

  // ---- per-cell update from / to shared memory ----
  if (kind != kSkip) {
    float f[27];
    load_tile<S>(sh, t, f);
    if (kind == kSolid) {
#pragma unroll
      for (int q = 1; q < 27; q += 2) {
        const float x = f[q];
        f[q] = f[q + 1];
        f[q + 1] = x;
      }
    } else {
      if (kind != kFluid) apply_boundary(m, f, p.given ? p.given[c0 + t] : p.given_uniform);
      collide<false>(f, p.rx);
      if (p.health) {
        const float r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6];
        if (!(r > 0.f && r < 1.0e30f)) atomicOr(p.health, 1u);
      }
    }
    store_tile<S>(sh, t, f);
  }
  fence_proxy_async_smem();
  __syncthreads();

  // ---- warp 0: write the row runs back ----
  if (t < 27) {
    T* row = p.g.fq[t];
    const T* srow = &sh.rows[t][0];
    const uint32_t a = shifted(c0, p.g.shift[t], n);
    const uint32_t s = (uint32_t)sh.off[t];
    if (a + kTile <= n) {
      write_segment<S>(row, srow, a, a + kTile, s);
    } else {
      write_segment<S>(row, srow, a, n, s);
      write_segment<S>(row, srow, 0, a + kTile - n, s + (n - a));
    }
    bulk_commit();
    bulk_wait_all();
  }
}

}  // namespace psl
