// Library-internal declarations shared by the C ABI translation units (psl_capi.cu,
// psl_batch.cu, psl_noalloc.cu): the grid object behind the opaque psl_grid handle and
// small host helpers.  Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "psl.h"

// Sets psl_last_error() for the calling thread (defined in psl_capi.cu).
__attribute__((visibility("hidden"))) void psl_detail_set_last_error(const std::string& msg);

// Make the grid's device current for the duration of a call, restoring the caller's.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------------------------------------
// grid
// ------------------------------------------------------------------------------------------
struct psl_grid {
  psl_info info;
  uint32_t n = 0;
  int storage = 0;
  size_t stride = 0;    // elements per per-cell array (markers, C_s, scalar rows): N rounded up to 64
  size_t f_stride = 0;  // elements from one population row of f to the next
  bool f_twice = false; // each population row mapped twice (psl_rowmap.cu): f_stride = 2N and
                        // row element N + i is element i, so the update needs no wrap
  struct psl_row_map* f_map = nullptr;  // the mappings when f_twice, else f is one cudaMalloc
  void* f = nullptr;
  uint8_t* marker = nullptr;
  float4* given = nullptr;
  float4 given_uniform = make_float4(1.f, 0.f, 0.f, 0.f);
  float cs = 0.f;
  float* cs_field = nullptr;        // per-cell Smagorinsky constants (getSmagorinskyConstant), or null
  uint32_t shift[27] = {};
  cudaStream_t stream = 0;
  unsigned int* health = nullptr;   // [0] health bits
  double* scratch = nullptr;        // force partials (kForceBlocks x 3) + result (3)
  int device = 0;
  int batched = 0;                  // member of this many live batches (psl_batch.cu)
  float3 body = make_float3(0.f, 0.f, 0.f);  // uniform body force (customised update)
  bool custom_markers = false;      // moving-wall or forced-velocity markers present
  float* T = nullptr;               // scalar-transport populations (27 FP32 rows), or null
  float* givenT = nullptr;          // per-cell prescribed concentration (NaN: none), or null
  float tauT = 1.f;
  void* mlp = nullptr;              // learned closure (psl::MlpDevice), or null: Smagorinsky
  float mlp_width = 1.f;            // filter width fed to the closure
  float mlp_scalars[24] = {};       // its normalisation, b3, output scale (psl::MlpScalars)
  int mlp_interval = 1;             // the closure runs on every mlp_interval-th update (16-bit storage)
  int mlp_since = 0;                // updates since its last run; 0: the next update runs it
  uint16_t* mlp_nut = nullptr;      // per-cell FP16 nu_t of its last run (mlp_interval > 1), or null
  // psl_update_grid's concurrent schedule (the coarse cells away from the refinement block
  // updated beside the fine updates and the transfer): a lowest-priority side stream for
  // those cells, a highest-priority stream for the fine updates and the transfer, and their
  // events, created on first use, or null
  cudaStream_t side = nullptr, hi = nullptr;
  cudaEvent_t ev_near = nullptr, ev_far = nullptr, ev_hi = nullptr;
};

// Marks the held nu_t of the learned closure as out of date, so that the next update
// evaluates the closure (after populations or markers were set from outside the update).
inline void psl_detail_closure_stale(psl_grid* g) { g->mlp_since = 0; }

// Thread-to-cell rotation of the update kernels (psl_capi.cu, cell_of_thread in
// psl_kernels.cuh).
__attribute__((visibility("hidden"))) uint32_t psl_detail_thread_rotation(const psl_grid* g);

// Launches the update kernel with the learned closure (psl_learned.cu); status as psl_*.
namespace psl {
struct ThreadRange;
}
__attribute__((visibility("hidden"))) int psl_detail_launch_learned(psl_grid* g, const psl::ThreadRange& range);

