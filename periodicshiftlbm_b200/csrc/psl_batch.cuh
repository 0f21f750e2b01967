// Batched update: many independent single-level grids (flow-past-sphere cases of uneven
// size and Reynolds number) advanced by ONE persistent kernel per step.
//
// Work decomposition: each case's cells are cut into tiles of `tile_cells` consecutive
// cells; the tiles of all cases form one index space that the resident warps walk with a
// fixed stride (warp w takes tiles w, w + warps, ...).  A table gives each tile's case; a
// small kernel before the update writes every case's 27 row offsets for the step, which
// lanes 0-26 copy into the warp's shared-memory slot at the start of a tile; every lane then
// updates cells of the tile exactly as the single-grid update kernel does
// (applyLocalCellUpdate.h:1-74).
//
// The periodic shifts are not kernel parameters: after s applications of applyStreaming
// (applyStreaming.h:11-31) the shift of population q is (shift0_q + s * adv_q) mod N with
// adv_q = -(c_x + N_x c_y + N_x N_y c_z) mod N, and the update of batch step s (counting
// from 0) runs on the shifts after s + 1 streamings, as updateGrid streams before it
// updates.  The step counter s lives in device memory.  So the launch sequence of one step -- the update
// kernel and the one-thread kernel that increments the counter -- is the same every step,
// and is captured once in a CUDA graph and replayed.
#pragma once
#include "psl_kernels.cuh"

namespace psl {

template <typename S>
struct BatchCase {
  typename S::type* f;    // base of the 27 population rows
  const uint8_t* marker;
  const float4* given;    // per-cell (rho, ux, uy, uz) for boundary cells, or null
  unsigned int* health;   // the grid's health word
  float4 given_uniform;
  RelaxationT<float> rx;
  uint32_t n;             // cells
  uint32_t stride;        // elements per population row
  uint32_t shift0[27];    // shifts at batch step 0
  uint32_t adv[27];       // per-step advance of each shift, in [0, n)
  uint32_t tile_begin;    // first tile of this case in the batch's tile space
};

constexpr int kBatchMaxThreads = 256;

// Rows of a tile that no population's wrap point cuts: population Q of `cell` is at
// base[cell + adj[Q]] with a tile-uniform adj (no per-cell compare).
template <typename S, int Q = 0>
__device__ __forceinline__ void load_cell_adj(typename S::type* base, const uint32_t (&adj)[27], uint32_t cell,
                                              float (&f)[27]) {
  if constexpr (Q < 27) {
    f[Q] = S::template load_once<Q>(base + (cell + adj[Q]));
    load_cell_adj<S, Q + 1>(base, adj, cell, f);
  }
}
template <typename S, int Q = 0>
__device__ __forceinline__ void store_cell_adj(typename S::type* base, const uint32_t (&adj)[27], uint32_t cell,
                                               const float (&f)[27]) {
  if constexpr (Q < 27) {
    S::template store_once<Q>(base + (cell + adj[Q]), f[Q]);
    store_cell_adj<S, Q + 1>(base, adj, cell, f);
  }
}

// Shift of population q at step `step`: (shift0 + step * adv) mod n, in 64-bit arithmetic
// (step mod n < 2^31 and adv < 2^31, so the product fits).
__device__ __forceinline__ uint32_t batch_shift(uint32_t shift0, uint32_t adv, uint32_t n, unsigned long long step) {
  const unsigned long long s = step % n;
  return (uint32_t)((s * adv + shift0) % n);
}

// Per step, before the update: every case's 27 row offsets and wrap limits for the shifts
// after step + 1 streamings (one block per case, one thread per population).
template <typename S>
__global__ void batch_offsets_kernel(const BatchCase<S>* __restrict__ cases, const unsigned long long* __restrict__ step,
                                     uint2* __restrict__ offsets) {
  const int c = blockIdx.x, q = threadIdx.x;
  if (q >= 27) return;
  const BatchCase<S>& bc = cases[c];
  const uint32_t sh = batch_shift(bc.shift0[q], bc.adv[q], bc.n, *step + 1);
  offsets[c * 27 + q] = make_uint2((uint32_t)q * bc.stride + sh, bc.n - sh);
}

// Warp tiles: every warp walks its own tiles of `tile_cells` consecutive cells (warp w of
// the grid takes tiles w, w + warps, ...) with its case data in its own shared-memory slot,
// so warps synchronise only within themselves (no CTA barrier couples them).
struct BatchWarpSlot {
  uint32_t off[27];
  uint32_t lim[27];
  uint32_t adj[27];  // tile-uniform offsets when no wrap point cuts the tile
};

template <typename S>
__global__ void __launch_bounds__(kBatchMaxThreads, 4) batch_step_kernel(const BatchCase<S>* __restrict__ cases,
                                                                         const uint32_t* __restrict__ tile_case,
                                                                         const uint2* __restrict__ offsets,
                                                                         uint32_t tiles, uint32_t tile_cells) {
  __shared__ BatchWarpSlot slots[kBatchMaxThreads / 32];
  const int lane = threadIdx.x & 31;
  BatchWarpSlot& slot = slots[threadIdx.x >> 5];
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t tile = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile < tiles; tile += warps) {
    const uint32_t ci = tile_case[tile];
    const BatchCase<S>& c = cases[ci];
    const uint32_t n = c.n;
    const uint32_t first = (tile - c.tile_begin) * tile_cells;
    const uint32_t last = min(first + tile_cells, n);
    bool cut = false;
    __syncwarp();  // the previous tile's readers of the slot are done
    if (lane < 27) {
      const uint2 ol = offsets[ci * 27 + lane];
      slot.off[lane] = ol.x;
      slot.lim[lane] = ol.y;
      slot.adj[lane] = ol.x - (first >= ol.y ? n : 0u);
      cut = first < ol.y && last - 1 >= ol.y;
    }
    const bool any_cut = __any_sync(0xffffffffu, cut);  // also orders the slot writes
    typename S::type* base = c.f;
    const uint8_t* marker = c.marker;
    for (uint32_t cell = first + lane; cell < last; cell += 32) {
      const uint8_t m = marker[cell];
      const int kind = marker_kind(m);
      if (kind == kSkip) continue;
      using V = StoredOf<S>;
      float f[27];
      if (!any_cut) {
        load_cell_adj<V>(base, slot.adj, cell, f);
      } else {
        RowIndex<V> ri;
        ri.base = base;
        ri.n = n;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
          ri.off[q] = slot.off[q];
          ri.lim[q] = slot.lim[q];
        }
        load_cell_ri<V>(ri, cell, f);
      }
      if constexpr (S::kind == kStoreF32) {
        local_cell_update<kBatchMaxThreads>(kind, m, f, c.given, c.given_uniform, cell, c.rx, c.health);
      } else if (kind == kSolid) {  // bounce-back swaps g as it swaps f (w_q = w_opposite(q))
#pragma unroll
        for (int q = 1; q < 27; q += 2) {
          const float t = f[q];
          f[q] = f[q + 1];
          f[q + 1] = t;
        }
      } else {
        __shared__ float bslot[kBatchMaxThreads][27];
        collide_cell_g(kind, m, f, c.given, c.given_uniform, cell, c.rx, c.rx.cs18, c.health, bslot[threadIdx.x]);
      }
      if (!any_cut) {
        store_cell_adj<V>(base, slot.adj, cell, f);
      } else {
        RowIndex<V> ri;
        ri.base = base;
        ri.n = n;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
          ri.off[q] = slot.off[q];
          ri.lim[q] = slot.lim[q];
        }
        store_cell_ri<V>(ri, cell, f);
      }
    }
  }
}

static __global__ void batch_advance_kernel(unsigned long long* step) { *step += 1; }

}  // namespace psl
