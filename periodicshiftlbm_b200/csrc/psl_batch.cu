// C ABI of the batched update (include/psl.h, "batched form"): a batch of independent
// single-level grids advanced by one kernel per step over all their tiles (psl_batch.cuh),
// the step captured once in a CUDA graph and replayed, and a project-written autotuner that
// picks the launch shape (threads per CTA, cells per warp tile, resident CTAs per SM or a
// one-pass grid) by timing candidates on the batch itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <set>
#include <string>
#include <vector>

#include "psl.h"
#include "psl_batch.cuh"
#include "psl_internal.h"

using namespace psl;

namespace {

int fail(int code, const std::string& msg) {
  psl_detail_set_last_error(msg);
  return code;
}

#define BATCH_CUDA(expr)                                                                               \
  do {                                                                                                 \
    cudaError_t e_ = (expr);                                                                           \
    if (e_ != cudaSuccess) return fail(PSL_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define BATCH_CHECK(cond, code, msg) \
  do {                               \
    if (!(cond)) return fail(code, msg); \
  } while (0)

// Per-step advance of each shift (applyStreaming.h:11-31): shift -= c_x + Nx c_y + Nx Ny c_z,
// as an addition in [0, n).
std::array<uint32_t, 27> shift_advance(const psl_grid* g) {
  std::array<uint32_t, 27> adv{};
  const long long nx = g->info.cell_count_x, ny = g->info.cell_count_y, n = g->n;
  for (int q = 0; q < 27; ++q) {
    long long d = cx(q) + nx * cy(q) + nx * ny * cz(q);
    long long a = (-d) % n;
    if (a < 0) a += n;
    adv[q] = (uint32_t)a;
  }
  return adv;
}

uint32_t shift_at(uint32_t shift0, uint32_t adv, uint32_t n, unsigned long long step) {
  return (uint32_t)(((step % n) * (unsigned long long)adv + shift0) % n);
}

}  // namespace

struct psl_batch {
  std::vector<psl_grid*> grids;
  int storage = 0;
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;    // owned, non-blocking
  cudaEvent_t done = nullptr;       // end of the last run, for the member grids' streams
  void* table = nullptr;            // device BatchCase<S>[count]
  unsigned long long* step = nullptr;  // device step counter
  unsigned long long steps_done = 0;   // host copy of the counter
  std::vector<std::array<uint32_t, 27>> shift0, adv;
  uint32_t tiles = 0;
  uint32_t* tile_case = nullptr;    // device: case of every tile
  uint2* offsets = nullptr;         // device: per case and population (offset, limit) of the step
  psl_batch_tuning tuning{};
  cudaGraphExec_t graph = nullptr;
  bool registered = false;          // counted in the member grids' `batched`
};

namespace {

template <typename S>
int occupancy(int threads, int* per_sm) {
  BATCH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_step_kernel<S>, threads, 0));
  return PSL_OK;
}

// Rebuild the device case table for the current tuning (the tile boundaries depend on
// tile_cells).  Stream-ordered on the batch stream.
template <typename S>
int upload_table(psl_batch* b) {
  std::vector<BatchCase<S>> host(b->grids.size());
  uint32_t tile = 0;
  const uint32_t tc = (uint32_t)b->tuning.tile_cells;
  for (size_t i = 0; i < b->grids.size(); ++i) {
    const psl_grid* g = b->grids[i];
    BatchCase<S>& c = host[i];
    c.f = static_cast<typename S::type*>(g->f);
    c.marker = g->marker;
    c.given = g->given;
    c.health = g->health;
    c.given_uniform = g->given_uniform;
    c.rx.tau = 3.f * g->info.nu + 0.5f;
    c.rx.tau2 = c.rx.tau * c.rx.tau;
    c.rx.omega0 = 1.f / c.rx.tau;
    c.rx.cs18 = 18.f * g->cs;
    c.n = g->n;
    c.stride = (uint32_t)g->f_stride;
    for (int q = 0; q < 27; ++q) {
      c.shift0[q] = b->shift0[i][q];
      c.adv[q] = b->adv[i][q];
    }
    c.tile_begin = tile;
    tile += (g->n + tc - 1) / tc;
  }
  b->tiles = tile;
  std::vector<uint32_t> case_of(tile);
  for (size_t i = 0; i < host.size(); ++i) {
    const uint32_t end = i + 1 < host.size() ? host[i + 1].tile_begin : tile;
    for (uint32_t t = host[i].tile_begin; t < end; ++t) case_of[t] = (uint32_t)i;
  }
  if (b->tile_case) cudaFree(b->tile_case);
  b->tile_case = nullptr;
  BATCH_CUDA(cudaMalloc(&b->tile_case, case_of.size() * sizeof(uint32_t)));
  BATCH_CUDA(cudaMemcpyAsync(b->tile_case, case_of.data(), case_of.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             b->stream));
  if (!b->offsets) BATCH_CUDA(cudaMalloc(&b->offsets, host.size() * 27 * sizeof(uint2)));
  if (!b->table) BATCH_CUDA(cudaMalloc(&b->table, host.size() * sizeof(BatchCase<S>)));
  BATCH_CUDA(cudaMemcpyAsync(b->table, host.data(), host.size() * sizeof(BatchCase<S>), cudaMemcpyHostToDevice,
                             b->stream));
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  return PSL_OK;
}

template <typename S>
void launch_one_step(psl_batch* b) {
  const int threads = b->tuning.threads;
  const unsigned int warps_per_block = (unsigned int)threads / 32;
  const unsigned int all_tiles = std::max(1u, (b->tiles + warps_per_block - 1) / warps_per_block);
  const unsigned int blocks =
      b->tuning.blocks_per_sm == 0 ? all_tiles
                                   : std::min(all_tiles, (unsigned int)(b->sms * b->tuning.blocks_per_sm));
  const BatchCase<S>* cases = static_cast<const BatchCase<S>*>(b->table);
  batch_offsets_kernel<S><<<(unsigned int)b->grids.size(), 32, 0, b->stream>>>(cases, b->step, b->offsets);
  batch_step_kernel<S><<<blocks, threads, 0, b->stream>>>(cases, b->tile_case, b->offsets, b->tiles,
                                                           (uint32_t)b->tuning.tile_cells);
  batch_advance_kernel<<<1, 1, 0, b->stream>>>(b->step);
}

template <typename Fn>
auto with_batch_storage(int storage, Fn&& fn) {
  switch (storage) {
    case kStoreF32: return fn(StoreF32{});
    case kStoreF16: return fn(StoreF16{});
    default: return fn(StoreBF16{});
  }
}

int drop_graph(psl_batch* b) {
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return PSL_OK;
}

int capture_graph(psl_batch* b) {
  cudaGraph_t graph = nullptr;
  BATCH_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  with_batch_storage(b->storage, [&](auto s) {
    launch_one_step<decltype(s)>(b);
    return 0;
  });
  cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    b->graph = nullptr;
    return fail(PSL_ERR_CUDA, std::string("psl_batch: graph capture: ") + cudaGetErrorString(e));
  }
  return PSL_OK;
}

int validate_tuning(const psl_batch* b, const psl_batch_tuning& t) {
  BATCH_CHECK(t.threads >= 32 && t.threads <= kBatchMaxThreads && t.threads % 32 == 0, PSL_ERR_INVALID,
              "psl_batch: threads must be a multiple of 32 in [32, 256]");
  BATCH_CHECK(t.tile_cells >= 32 && t.tile_cells % 32 == 0 && t.tile_cells <= (1 << 20), PSL_ERR_INVALID,
              "psl_batch: tile_cells (cells per warp tile) must be a multiple of 32, at most 2^20");
  BATCH_CHECK(t.blocks_per_sm >= 0 && t.blocks_per_sm <= 64, PSL_ERR_INVALID, "psl_batch: blocks_per_sm out of range");
  int per_sm = 0;
  int rc = with_batch_storage(b->storage, [&](auto s) { return occupancy<decltype(s)>(t.threads, &per_sm); });
  if (rc) return rc;
  BATCH_CHECK(t.blocks_per_sm <= per_sm, PSL_ERR_INVALID, "psl_batch: more CTAs per SM than can be resident");
  return PSL_OK;
}

int apply_tuning(psl_batch* b, const psl_batch_tuning& t) {
  int rc = validate_tuning(b, t);
  if (rc) return rc;
  b->tuning = t;
  drop_graph(b);
  return with_batch_storage(b->storage, [&](auto s) { return upload_table<decltype(s)>(b); });
}

// Make the batch stream wait for work queued on the member grids' streams.
int wait_for_members(psl_batch* b) {
  std::set<cudaStream_t> streams;
  for (psl_grid* g : b->grids) streams.insert(g->stream);
  for (cudaStream_t s : streams) BATCH_CUDA(cudaStreamSynchronize(s));
  return PSL_OK;
}

// Bring the member grids' host shifts to the batch step and order their streams after the
// batch's work.
int publish(psl_batch* b) {
  for (size_t i = 0; i < b->grids.size(); ++i) {
    psl_grid* g = b->grids[i];
    for (int q = 0; q < 27; ++q) g->shift[q] = shift_at(b->shift0[i][q], b->adv[i][q], g->n, b->steps_done);
  }
  BATCH_CUDA(cudaEventRecord(b->done, b->stream));
  std::set<cudaStream_t> streams;
  for (psl_grid* g : b->grids) streams.insert(g->stream);
  for (cudaStream_t s : streams) BATCH_CUDA(cudaStreamWaitEvent(s, b->done, 0));
  return PSL_OK;
}

}  // namespace

int psl_batch_create(psl_grid* const* grids, int count, psl_batch** out) {
  BATCH_CHECK(grids && out && count > 0, PSL_ERR_INVALID, "psl_batch_create: bad argument");
  *out = nullptr;
  std::set<const psl_grid*> seen;
  for (int i = 0; i < count; ++i) {
    const psl_grid* g = grids[i];
    BATCH_CHECK(g, PSL_ERR_INVALID, "psl_batch_create: null grid");
    BATCH_CHECK(seen.insert(g).second, PSL_ERR_INVALID, "psl_batch_create: a grid appears twice");
    BATCH_CHECK(g->device == grids[0]->device, PSL_ERR_INVALID, "psl_batch_create: grids on different devices");
    BATCH_CHECK(g->storage == grids[0]->storage, PSL_ERR_INVALID, "psl_batch_create: grids use different storage");
    BATCH_CHECK(g->storage != kStoreF64, PSL_ERR_INVALID, "psl_batch_create: FP64 storage is for oracle runs only");
    BATCH_CHECK(g->info.i_subgrid_end <= g->info.i_subgrid_start, PSL_ERR_INVALID,
                "psl_batch_create: grids with a refinement block are not batched");
    BATCH_CHECK(27ull * g->f_stride + g->n < (1ull << 32), PSL_ERR_INVALID, "psl_batch_create: grid too large");
    BATCH_CHECK(!g->cs_field, PSL_ERR_INVALID,
                "psl_batch_create: grids with a per-cell Smagorinsky field are not batched");
  }
  DeviceGuard dg(grids[0]->device);
  psl_batch* b = new psl_batch();
  b->grids.assign(grids, grids + count);
  b->storage = grids[0]->storage;
  b->device = grids[0]->device;
  for (psl_grid* g : b->grids) {
    std::array<uint32_t, 27> s0{};
    for (int q = 0; q < 27; ++q) s0[q] = g->shift[q];
    b->shift0.push_back(s0);
    b->adv.push_back(shift_advance(g));
  }
  cudaError_t e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->step, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(b->step, 0, sizeof(unsigned long long), b->stream);
  if (e != cudaSuccess) {
    const std::string msg = std::string("psl_batch_create: ") + cudaGetErrorString(e);
    cudaGetLastError();
    psl_batch_destroy(b);
    return fail(e == cudaErrorMemoryAllocation ? PSL_ERR_NOMEM : PSL_ERR_CUDA, msg);
  }
  psl_batch_tuning t{};
  t.threads = 128;
  t.tile_cells = 256;
  int per_sm = 0;
  int rc = with_batch_storage(b->storage, [&](auto s) { return occupancy<decltype(s)>(t.threads, &per_sm); });
  t.blocks_per_sm = std::max(1, per_sm);
  if (!rc) rc = apply_tuning(b, t);
  if (rc) {
    psl_batch_destroy(b);
    return rc;
  }
  for (psl_grid* g : b->grids) g->batched += 1;
  b->registered = true;
  *out = b;
  return PSL_OK;
}

int psl_batch_destroy(psl_batch* b) {
  if (!b) return PSL_OK;
  DeviceGuard dg(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  if (b->table) cudaFree(b->table);
  if (b->tile_case) cudaFree(b->tile_case);
  if (b->offsets) cudaFree(b->offsets);
  if (b->step) cudaFree(b->step);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->registered)
    for (psl_grid* g : b->grids) g->batched -= 1;
  delete b;
  return PSL_OK;
}

int psl_batch_get_tuning(const psl_batch* b, psl_batch_tuning* t) {
  BATCH_CHECK(b && t, PSL_ERR_INVALID, "psl_batch_get_tuning: null argument");
  *t = b->tuning;
  return PSL_OK;
}

int psl_batch_set_tuning(psl_batch* b, const psl_batch_tuning* t) {
  BATCH_CHECK(b && t, PSL_ERR_INVALID, "psl_batch_set_tuning: null argument");
  DeviceGuard dg(b->device);
  return apply_tuning(b, *t);
}

int psl_batch_get_stream(const psl_batch* b, void** stream) {
  BATCH_CHECK(b && stream, PSL_ERR_INVALID, "psl_batch_get_stream: null argument");
  *stream = b->stream;
  return PSL_OK;
}

int psl_batch_run(psl_batch* b, int steps) {
  BATCH_CHECK(b && steps >= 0, PSL_ERR_INVALID, "psl_batch_run: bad argument");
  DeviceGuard dg(b->device);
  for (size_t i = 0; i < b->grids.size(); ++i)
    for (int q = 0; q < 27; ++q)
      BATCH_CHECK(b->grids[i]->shift[q] == shift_at(b->shift0[i][q], b->adv[i][q], b->grids[i]->n, b->steps_done),
                  PSL_ERR_INVALID, "psl_batch_run: a member grid was streamed outside the batch");
  int rc = wait_for_members(b);
  if (rc) return rc;
  if (!b->graph) {
    rc = capture_graph(b);
    if (rc) return rc;
  }
  for (int s = 0; s < steps; ++s) BATCH_CUDA(cudaGraphLaunch(b->graph, b->stream));
  b->steps_done += (unsigned long long)steps;
  return publish(b);
}

int psl_batch_synchronize(psl_batch* b) {
  BATCH_CHECK(b, PSL_ERR_INVALID, "psl_batch_synchronize: null batch");
  DeviceGuard dg(b->device);
  BATCH_CUDA(cudaStreamSynchronize(b->stream));
  return PSL_OK;
}

int psl_batch_autotune(psl_batch* b, int trial_steps, psl_batch_tuning* chosen) {
  BATCH_CHECK(b && trial_steps > 0, PSL_ERR_INVALID, "psl_batch_autotune: bad argument");
  DeviceGuard dg(b->device);
  int rc = wait_for_members(b);
  if (rc) return rc;
  // save the populations (and the step counter) so tuning leaves the simulation unchanged
  std::vector<void*> saved(b->grids.size(), nullptr);
  std::vector<size_t> bytes(b->grids.size());
  auto release = [&]() {
    for (void* p : saved)
      if (p) cudaFree(p);
  };
  for (size_t i = 0; i < b->grids.size(); ++i) {
    const psl_grid* g = b->grids[i];
    // rows of N values each (f's rows may be mapped twice: copy one mapping)
    bytes[i] = (size_t)g->n * storage_bytes(g->storage);
    cudaError_t e = cudaMalloc(&saved[i], 27 * bytes[i]);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(saved[i], bytes[i], g->f, g->f_stride * storage_bytes(g->storage), bytes[i], 27,
                            cudaMemcpyDeviceToDevice, b->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      release();
      return fail(e == cudaErrorMemoryAllocation ? PSL_ERR_NOMEM : PSL_ERR_CUDA,
                  std::string("psl_batch_autotune: saving the state: ") + cudaGetErrorString(e));
    }
  }
  const psl_batch_tuning original = b->tuning;
  psl_batch_tuning best = original;
  best.ms_per_step = 1e30f;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int thread_options[] = {64, 128, 256};
  const int tile_factors[] = {1, 2, 4, 8, 16, 32};  // warp tiles of 32 x factor cells
  for (int threads : thread_options) {
    int per_sm = 0;
    rc = with_batch_storage(b->storage, [&](auto s) { return occupancy<decltype(s)>(threads, &per_sm); });
    if (rc || per_sm < 1) continue;
    // resident grids of per_sm and per_sm/2 CTAs per SM, and (0) one CTA per tiles' worth
    const int resident[] = {per_sm, std::max(1, per_sm / 2), 0};
    for (int r = 0; r < 3; ++r)
      for (int tf : tile_factors) {
        psl_batch_tuning t{};
        t.threads = threads;
        t.tile_cells = 32 * tf;
        t.blocks_per_sm = resident[r];
        if (apply_tuning(b, t)) continue;
        with_batch_storage(b->storage, [&](auto s) {
          launch_one_step<decltype(s)>(b);  // warm-up
          cudaEventRecord(t0, b->stream);
          for (int k = 0; k < trial_steps; ++k) launch_one_step<decltype(s)>(b);
          cudaEventRecord(t1, b->stream);
          return 0;
        });
        float ms = 0.f;
        if (cudaEventSynchronize(t1) != cudaSuccess || cudaEventElapsedTime(&ms, t0, t1) != cudaSuccess) continue;
        t.ms_per_step = ms / trial_steps;
        if (t.ms_per_step < best.ms_per_step) best = t;
      }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  // restore the state and the counter, then adopt the winner
  for (size_t i = 0; i < b->grids.size(); ++i)
    cudaMemcpy2DAsync(b->grids[i]->f, b->grids[i]->f_stride * storage_bytes(b->grids[i]->storage), saved[i], bytes[i],
                      bytes[i], 27, cudaMemcpyDeviceToDevice, b->stream);
  cudaMemcpyAsync(b->step, &b->steps_done, sizeof(unsigned long long), cudaMemcpyHostToDevice, b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  release();
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_batch_autotune: ") + cudaGetErrorString(e));
  cudaGetLastError();
  if (best.ms_per_step >= 1e30f) {
    apply_tuning(b, original);
    return fail(PSL_ERR_CUDA, "psl_batch_autotune: no candidate ran");
  }
  rc = apply_tuning(b, best);
  b->tuning.ms_per_step = best.ms_per_step;
  if (chosen) *chosen = b->tuning;
  return rc;
}
