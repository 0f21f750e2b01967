// Thread-to-cell order of the update kernels that keeps the x-face cells in warps of their
// own.
//
// In cell order (i fastest) every x-row starts and ends with an x-face cell: the inflow and
// outflow planes of the sphere cases (given velocity / given density), the ghost layer of a
// fine grid.  With one thread per cell in that order, the warp holding cell i = 0 and the
// warp holding i = Nx - 1 of each row carry one boundary cell among 31 fluid cells and run
// both the fluid path and the boundary branch: on the 512-wide coarse grid of the sphere
// case that is one warp in eight, ~7% of the FP16 launch.  The grouped order takes the rows
// sixteen at a time: the group's 16 (Nx - 2) interior cells in cell order first (whole warps
// when Nx is even; a warp crosses a row end with a two-cell gap, still one coalesced run),
// then its 32 x-face cells in one warp, ordered (row r, 0), (row r, Nx - 1), (row r + 1, 0),
// ..., so that the end of one row and the start of the next sit in neighbouring lanes.  The
// x-face warp runs next to the interior warps of the same rows, whose loads have just brought
// the shared sectors into L2.  A bijection of [0, N): every cell is updated exactly once, as
// in cell order.
#pragma once
#include <stdint.h>

#include "psl_lattice.cuh"

namespace psl {

// Unsigned division by a run-time constant d >= 1 (round-up multiplier, exact for every
// 32-bit dividend: Granlund & Montgomery 1994, section 4): q = (t + ((x - t) >> 1)) >> (l - 1)
// with t = mulhi(m, x), l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1.
struct FastDiv {
  uint32_t d = 1, m = 0, s = 0;  // s = l - 1 (l >= 1); d == 1 handled apart
  FastDiv() = default;
  explicit FastDiv(uint32_t div) : d(div) {
    uint32_t l = 0;
    while (l < 32 && (1ull << l) < div) ++l;
    m = (uint32_t)(((1ull << 32) * ((1ull << l) - div)) / div + 1);
    s = l ? l - 1 : 0;
  }
  PSL_HDI uint32_t div(uint32_t x) const {
    if (d == 1) return x;
#if defined(__CUDA_ARCH__)
    const uint32_t t = __umulhi(m, x);
#else
    const uint32_t t = (uint32_t)(((uint64_t)m * x) >> 32);
#endif
    return (t + ((x - t) >> 1)) >> s;
  }
};

struct RowGroups {
  uint32_t nx = 0;          // cells per x-row (even, >= 4)
  uint32_t rows = 0;        // x-rows of the grid (Ny Nz)
  FastDiv by_nx;            // t / Nx, t < 2^32
  FastDiv by_inner;         // v / (Nx - 2)
};

inline RowGroups make_row_groups(uint32_t nx, uint32_t rows) {
  RowGroups g;
  g.nx = nx;
  g.rows = rows;
  g.by_nx = FastDiv(nx);
  g.by_inner = FastDiv(nx - 2);
  return g;
}

// Cell updated by thread t (t < Nx rows) in the grouped order.
PSL_HDI uint32_t grouped_cell(uint32_t t, const RowGroups& g) {
  const uint32_t group = g.by_nx.div(t >> 4);               // t / (16 Nx)
  const uint32_t first_row = group * 16u;
  const uint32_t rows = g.rows - first_row < 16u ? g.rows - first_row : 16u;
  const uint32_t v = t - first_row * g.nx;                  // position in the group
  const uint32_t inner = g.nx - 2u;
  if (v < rows * inner) {
    const uint32_t r = g.by_inner.div(v);
    return (first_row + r) * g.nx + 1u + (v - r * inner);
  }
  // x-face lanes: w = 2r is (row r, 0), w = 2r + 1 is (row r, Nx - 1); lanes 2r + 1 and
  // 2r + 2 hold neighbouring cells (the end of row r, the start of row r + 1)
  const uint32_t w = v - rows * inner;
  return (first_row + (w >> 1)) * g.nx + ((w & 1u) ? g.nx - 1u : 0u);
}

}  // namespace psl
