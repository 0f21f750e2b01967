// Batched update: many independent single-level grids (flow-past-sphere cases of uneven
// size and Reynolds number) advanced by ONE persistent kernel per step.
//
// Work decomposition: each case's cells are cut into tiles of `tile_cells` consecutive
// cells; the tiles of all cases form one index space that a grid of resident CTAs walks
// with a fixed stride (CTA b takes tiles b, b + gridDim, ...).  At the start of a tile the
// CTA finds the tile's case (binary search over the cases' first tiles), and threads 0-26
// derive the case's 27 row offsets for the current step into shared memory; every thread
// then updates cells of the tile exactly as the single-grid update kernel does
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

// Shift of population q at step `step`: (shift0 + step * adv) mod n, in 64-bit arithmetic
// (step mod n < 2^31 and adv < 2^31, so the product fits).
__device__ __forceinline__ uint32_t batch_shift(uint32_t shift0, uint32_t adv, uint32_t n, unsigned long long step) {
  const unsigned long long s = step % n;
  return (uint32_t)((s * adv + shift0) % n);
}

template <typename S>
__global__ void __launch_bounds__(kBatchMaxThreads) batch_step_kernel(const BatchCase<S>* __restrict__ cases, int ncases,
                                                                      uint32_t tiles, uint32_t tile_cells,
                                                                      const unsigned long long* __restrict__ step) {
  // the current tile's case: row offsets and scalars live in shared memory, so the cell
  // loop holds no per-case registers
  __shared__ RowIndex<S> ri;
  __shared__ int s_case;
  __shared__ RelaxationT<float> s_rx;
  __shared__ float4 s_given_uniform;
  __shared__ const uint8_t* s_marker;
  __shared__ const float4* s_given;
  __shared__ unsigned int* s_health;
  const unsigned long long st = *step;
  for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    __syncthreads();  // the previous tile's readers of `ri` are done
    if (threadIdx.x < 27) {
      int lo = 0, hi = ncases - 1;  // last case whose first tile is <= tile
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cases[mid].tile_begin <= tile) lo = mid;
        else hi = mid - 1;
      }
      const BatchCase<S>& c = cases[lo];
      const int q = threadIdx.x;
      const uint32_t sh = batch_shift(c.shift0[q], c.adv[q], c.n, st + 1);
      ri.off[q] = (uint32_t)q * c.stride + sh;
      ri.lim[q] = c.n - sh;
      if (q == 0) {
        ri.base = c.f;
        ri.n = c.n;
        s_case = lo;
        s_rx = c.rx;
        s_given_uniform = c.given_uniform;
        s_marker = c.marker;
        s_given = c.given;
        s_health = c.health;
      }
    }
    __syncthreads();
    const uint32_t first = (tile - cases[s_case].tile_begin) * tile_cells;
    const uint32_t last = min(first + tile_cells, ri.n);
    for (uint32_t cell = first + threadIdx.x; cell < last; cell += blockDim.x) {
      const uint8_t m = s_marker[cell];
      const int kind = marker_kind(m);
      if (kind == kSkip) continue;
      float f[27];
      load_cell_ri<S>(ri, cell, f);
      local_cell_update(kind, m, f, s_given, s_given_uniform, cell, s_rx, s_health);
      store_cell_ri<S>(ri, cell, f);
    }
  }
}

static __global__ void batch_advance_kernel(unsigned long long* step) { *step += 1; }

}  // namespace psl
