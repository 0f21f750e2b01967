// Host build of the grouped thread-to-cell order (periodicshiftlbm_b200/csrc/psl_rowgroups.cuh)
// for the CPU tests: the fast division and the permutation.
#include <stdint.h>

#include "psl_rowgroups.cuh"

extern "C" uint32_t fastdiv_host(uint32_t d, uint32_t x) { return psl::FastDiv(d).div(x); }

extern "C" void grouped_cells_host(uint32_t nx, uint32_t rows, uint32_t* out) {
  const psl::RowGroups g = psl::make_row_groups(nx, rows);
  for (uint32_t t = 0; t < nx * rows; ++t) out[t] = psl::grouped_cell(t, g);
}
