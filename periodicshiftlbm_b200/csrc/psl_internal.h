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
  size_t stride = 0;  // elements per population row, multiple of 64 (128-byte rows)
  void* f = nullptr;
  uint8_t* marker = nullptr;
  float4* given = nullptr;
  float4 given_uniform = make_float4(1.f, 0.f, 0.f, 0.f);
  float cs = 0.f;
  float* cs_field = nullptr;        // per-cell Smagorinsky constants (getSmagorinskyConstant), or null
  // Capture of the x-face ring cells' children for the coarse/fine restriction (a fine
  // grid's update writes it, Capture in psl_kernels.cuh): allocated by the first transfer,
  // used while the fine grid's last population change was a capturing update.
  void* xcap = nullptr;
  int xcap_i0 = 0, xcap_i1 = 0;     // first fine column of each captured pair
  unsigned long long state_version = 0;  // bumped by every call that changes the populations
  unsigned long long xcap_version = 0;   // state_version the capture belongs to
  uint32_t shift[27] = {};
  cudaStream_t stream = 0;
  unsigned int* health = nullptr;   // [0] health bits, [1] barrier counter
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
};

// Every call that changes a grid's populations or shifts calls this first.
inline void psl_detail_touch(psl_grid* g) { ++g->state_version; }

// The capture a fine grid's update writes for the coarse/fine restriction (Capture<S>,
// psl_kernels.cuh; buf null when the grid has none); marks the grid's current state as
// captured.  The row of a cell is cell / Nx by multiply-shift: s = 31 + ceil(log2 Nx),
// m = floor(2^s / Nx) + 1, exact for every cell < 2^31.
template <typename C>
inline void psl_detail_fill_capture(psl_grid* g, C& cap) {
  cap.buf = static_cast<decltype(cap.buf)>(g->xcap);
  cap.nx = (uint32_t)g->info.cell_count_x;
  cap.rows = (uint32_t)g->info.cell_count_y * (uint32_t)g->info.cell_count_z;
  cap.i0 = (uint32_t)g->xcap_i0;
  cap.i1 = (uint32_t)g->xcap_i1;
  uint32_t log2_nx = 0;
  while ((1ull << log2_nx) < cap.nx) ++log2_nx;
  cap.div_s = 31 + log2_nx;
  cap.div_m = ((1ull << cap.div_s) / cap.nx) + 1;
  if (g->xcap) g->xcap_version = g->state_version;
}

// Launches the update kernel with the learned closure (psl_learned.cu); status as psl_*.
__attribute__((visibility("hidden"))) int psl_detail_launch_learned(psl_grid* g);

