// Population rows mapped twice in virtual memory (psl_rowmap.cu).  Library-internal.
#pragma once
#include <cuda_runtime.h>

#include <string>

struct psl_row_map;

// Allocates `rows` rows of `row_bytes` each on `device`, row r mapped at
// base + 2 r row_bytes and again at base + (2 r + 1) row_bytes.  Returns cudaSuccess,
// cudaErrorNotSupported when the driver or the row size does not allow it (nothing
// allocated; `why` says which), or the allocation error.
__attribute__((visibility("hidden"))) cudaError_t psl_row_map_create(int device, size_t row_bytes, int rows,
                                                                     void** base, psl_row_map** out,
                                                                     std::string* why);
__attribute__((visibility("hidden"))) void psl_row_map_destroy(psl_row_map* map);
