// C ABI of the lattice update (include/psl.h): grid handles, set-up, per-step launches,
// reductions and data movement.  Host-side logic only; the kernels are in psl_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "psl.h"
#include "psl_internal.h"
#include "psl_kernels.cuh"
#include "psl_rowmap.h"

using namespace psl;

// ------------------------------------------------------------------------------------------
// errors
// ------------------------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

// For the library's other translation units (psl_noalloc.cu).
__attribute__((visibility("hidden"))) void psl_detail_set_last_error(const std::string& msg) { g_last_error = msg; }

#define PSL_CUDA(expr)                                                                                 \
  do {                                                                                                 \
    cudaError_t e_ = (expr);                                                                           \
    if (e_ != cudaSuccess) return fail(PSL_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define PSL_CHECK(cond, code, msg) \
  do {                             \
    if (!(cond)) return fail(code, msg); \
  } while (0)

static constexpr int kForceBlocks = 512;

template <typename S>
static GridView<S> view(const psl_grid* g) {
  GridView<S> v;
  typename S::type* base = static_cast<typename S::type*>(g->f);
  for (int q = 0; q < 27; ++q) {
    v.fq[q] = base + (size_t)q * g->f_stride;
    v.shift[q] = g->shift[q];
  }
  v.n = g->n;
  return v;
}

// Base pointer + 32-bit row offsets of a grid's populations (needs 27 f_stride + N < 2^32).
template <typename S>
static RowIndex<S> row_index(const psl_grid* g) {
  RowIndex<S> r;
  r.base = static_cast<typename S::type*>(g->f);
  r.n = g->n;
  for (int q = 0; q < 27; ++q) {
    r.off[q] = (uint32_t)((size_t)q * g->f_stride + g->shift[q]);
    r.lim[q] = g->n - g->shift[q];
  }
  return r;
}

static InfoStruct hook_info(const psl_grid* g) {
  InfoStruct I;
  I.gridID = (float)g->info.grid_id;
  I.res = g->info.res;
  I.cellCountX = g->info.cell_count_x;
  I.cellCountY = g->info.cell_count_y;
  I.cellCountZ = g->info.cell_count_z;
  I.cellCount = (int)g->n;
  I.ox = g->info.ox;
  I.oy = g->info.oy;
  I.oz = g->info.oz;
  I.nu = g->info.nu;
  I.dtPhys = g->info.dt_phys;
  I.iSubgridStart = g->info.i_subgrid_start;
  I.jSubgridStart = g->info.j_subgrid_start;
  I.kSubgridStart = g->info.k_subgrid_start;
  I.iSubgridEnd = g->info.i_subgrid_end;
  I.jSubgridEnd = g->info.j_subgrid_end;
  I.kSubgridEnd = g->info.k_subgrid_end;
  return I;
}

static SphereCase sphere_hooks(const psl_sphere_case* sc) {
  SphereCase c;
  c.sx = sc->sphere_x;
  c.sy = sc->sphere_y;
  c.sz = sc->sphere_z;
  c.r = sc->sphere_r;
  c.uIn = sc->u_in;
  c.rhoGiven = sc->rho_given;
  c.wallMode = sc->wall_mode;
  c.smagorinsky = sc->smagorinsky;
  c.seed = sc->seed;
  c.noiseAmp = sc->noise_amp;
  return c;
}

static unsigned int blocks_for(size_t n, int threads) { return (unsigned int)((n + threads - 1) / threads); }

// Calls fn with a value of the grid's storage type (StoreF32 / StoreF16 / StoreBF16 /
// StoreF64) and returns what it returns.
template <typename Fn>
static auto with_storage(int storage, Fn&& fn) {
  switch (storage) {
    case kStoreF32: return fn(StoreF32{});
    case kStoreF16: return fn(StoreF16{});
    case kStoreBF16: return fn(StoreBF16{});
    default: return fn(StoreF64{});
  }
}

// Every psl_* definition below takes C linkage from its declaration in psl.h.

const char* psl_last_error(void) { return g_last_error.c_str(); }
const char* psl_version(void) { return "periodicshiftlbm_b200 0.1 (sm_100a)"; }

int psl_grid_create(const psl_info* info, int storage, psl_grid** out) {
  return psl_grid_create_ex(info, storage, 0u, out);
}

int psl_grid_create_ex(const psl_info* info, int storage, unsigned int flags, psl_grid** out) {
  PSL_CHECK(info && out, PSL_ERR_INVALID, "psl_grid_create: null argument");
  PSL_CHECK((flags & ~(unsigned int)PSL_GRID_ONE_MAPPING) == 0, PSL_ERR_INVALID, "psl_grid_create: unknown flags");
  *out = nullptr;
  const long long nx = info->cell_count_x, ny = info->cell_count_y, nz = info->cell_count_z;
  PSL_CHECK(nx > 0 && ny > 0 && nz > 0, PSL_ERR_INVALID, "psl_grid_create: cell counts must be positive");
  const long long n = nx * ny * nz;
  // the reference's shift normalisation (applyStreaming.h:24-27) wraps at most twice,
  // which covers every grid except Ny = Nz = 1
  PSL_CHECK(!(ny == 1 && nz == 1), PSL_ERR_INVALID, "psl_grid_create: Ny = Nz = 1 grids are not supported");
  PSL_CHECK(n < (1LL << 31), PSL_ERR_INVALID, "psl_grid_create: more than 2^31-1 cells");
  PSL_CHECK(storage >= 0 && storage <= 3, PSL_ERR_INVALID, "psl_grid_create: unknown storage");
  const bool has_block = info->i_subgrid_end > info->i_subgrid_start;
  if (has_block) {
    PSL_CHECK(info->i_subgrid_start >= 0 && info->i_subgrid_end <= nx && info->j_subgrid_start >= 0 &&
                  info->j_subgrid_end <= ny && info->k_subgrid_start >= 0 && info->k_subgrid_end <= nz,
              PSL_ERR_INVALID, "psl_grid_create: refinement block outside the grid");
  }
  int ndev = 0;
  PSL_CUDA(cudaGetDeviceCount(&ndev));
  PSL_CHECK(ndev > 0, PSL_ERR_CUDA, "psl_grid_create: no CUDA device");
  psl_grid* g = new psl_grid();
  g->info = *info;
  g->n = (uint32_t)n;
  g->storage = storage;
  g->stride = ((size_t)n + 63) / 64 * 64;
  cudaGetDevice(&g->device);
  const size_t elem = storage_bytes(storage);
  // population rows mapped twice where the row size allows it (psl_rowmap.cu), else one
  // allocation of 27 rows of `stride` elements
  cudaError_t e = cudaErrorNotSupported;
  const bool flat_fits = 55ull * (unsigned long long)n < (1ull << 32);  // 32-bit offsets of 27 rows of 2N, + N
  if (!(flags & PSL_GRID_ONE_MAPPING) && flat_fits)
    e = psl_row_map_create(g->device, (size_t)n * elem, 27, &g->f, &g->f_map, nullptr);
  if (e == cudaSuccess) {
    g->f_twice = true;
    g->f_stride = 2 * (size_t)n;
  } else {
    cudaGetLastError();
    g->f_stride = g->stride;
    e = cudaMalloc(&g->f, 27 * g->stride * elem);
  }
  if (e == cudaSuccess) e = cudaMalloc(&g->marker, g->stride);
  if (e == cudaSuccess) e = cudaMalloc(&g->health, 4 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&g->scratch, (kForceBlocks * 3 + 3) * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(g->marker, make_marker(kFluid, 0), g->stride);
  if (e == cudaSuccess) e = cudaMemset(g->health, 0, 4 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset2D(g->f, g->f_stride * elem, 0, (g->f_twice ? (size_t)n : g->stride) * elem, 27);
  if (e != cudaSuccess) {
    const std::string msg = std::string("psl_grid_create: ") + cudaGetErrorString(e);
    psl_grid_destroy(g);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? PSL_ERR_NOMEM : PSL_ERR_CUDA, msg);
  }
  *out = g;
  return PSL_OK;
}

int psl_grid_destroy(psl_grid* g) {
  if (!g) return PSL_OK;
  PSL_CHECK(g->batched == 0, PSL_ERR_INVALID, "psl_grid_destroy: the grid belongs to a live batch");
  DeviceGuard dg(g->device);
  if (g->f_map) psl_row_map_destroy(g->f_map);
  else if (g->f) cudaFree(g->f);
  if (g->marker) cudaFree(g->marker);
  if (g->given) cudaFree(g->given);
  if (g->health) cudaFree(g->health);
  if (g->scratch) cudaFree(g->scratch);
  if (g->mlp) cudaFree(g->mlp);
  if (g->T) cudaFree(g->T);
  if (g->givenT) cudaFree(g->givenT);
  if (g->cs_field) cudaFree(g->cs_field);
  if (g->mlp_nut) cudaFree(g->mlp_nut);
  for (cudaStream_t s : {g->side, g->hi}) {
    if (!s) continue;
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : {g->ev_near, g->ev_far, g->ev_hi})
    if (e) cudaEventDestroy(e);
  delete g;
  return PSL_OK;
}

int psl_grid_get_layout(const psl_grid* g, int* rows_mapped_twice, long long* row_stride) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_grid_get_layout: null grid");
  if (rows_mapped_twice) *rows_mapped_twice = g->f_twice ? 1 : 0;
  if (row_stride) *row_stride = (long long)g->f_stride;
  return PSL_OK;
}

int psl_grid_set_stream(psl_grid* g, void* stream) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_grid_set_stream: null grid");
  g->stream = static_cast<cudaStream_t>(stream);
  return PSL_OK;
}

int psl_grid_get_info(const psl_grid* g, psl_info* info, long long* cell_count, int* storage) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_grid_get_info: null grid");
  if (info) *info = g->info;
  if (cell_count) *cell_count = g->n;
  if (storage) *storage = g->storage;
  return PSL_OK;
}

// ---- hooks ----
int psl_apply_sphere_case(psl_grid* g, const psl_sphere_case* sc) {
  PSL_CHECK(g && sc, PSL_ERR_INVALID, "psl_apply_sphere_case: null argument");
  psl_detail_closure_stale(g);
  DeviceGuard dg(g->device);
  fill_markers_kernel<SphereCase><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(sphere_hooks(sc), hook_info(g), g->n,
                                                                                 g->marker, nullptr);
  PSL_CUDA(cudaGetLastError());
  g->given_uniform = make_float4(sc->rho_given, sc->u_in, 0.f, 0.f);
  g->cs = sc->smagorinsky;
  return PSL_OK;
}

int psl_set_markers(psl_grid* g, const uint8_t* host) {
  PSL_CHECK(g && host, PSL_ERR_INVALID, "psl_set_markers: null argument");
  psl_detail_closure_stale(g);
  DeviceGuard dg(g->device);
  // moving walls (solid, normal bits 1) and forced-velocity cells (fluid, normal bits 1)
  // select the customised update kernel
  g->custom_markers = false;
  for (uint32_t c = 0; c < g->n && !g->custom_markers; ++c) {
    const int kind = marker_kind(host[c]);
    g->custom_markers = (kind == kSolid || kind == kFluid) && marker_normal(host[c]) == 1;
  }
  PSL_CUDA(cudaMemcpyAsync(g->marker, host, g->n, cudaMemcpyHostToDevice, g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_get_markers(psl_grid* g, uint8_t* host) {
  PSL_CHECK(g && host, PSL_ERR_INVALID, "psl_get_markers: null argument");
  DeviceGuard dg(g->device);
  PSL_CUDA(cudaMemcpyAsync(host, g->marker, g->n, cudaMemcpyDeviceToHost, g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_set_given(psl_grid* g, float rho, float ux, float uy, float uz) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_given: null grid");
  g->given_uniform = make_float4(rho, ux, uy, uz);
  return PSL_OK;
}

int psl_set_given_field(psl_grid* g, const float* host) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_given_field: null grid");
  DeviceGuard dg(g->device);
  if (!host) {
    if (g->given) {
      PSL_CUDA(cudaStreamSynchronize(g->stream));
      cudaFree(g->given);
      g->given = nullptr;
    }
    return PSL_OK;
  }
  if (!g->given) {
    cudaError_t e = cudaMalloc(&g->given, (size_t)g->n * sizeof(float4));
    if (e != cudaSuccess) {
      g->given = nullptr;
      cudaGetLastError();
      return fail(PSL_ERR_NOMEM, std::string("psl_set_given_field: ") + cudaGetErrorString(e));
    }
  }
  PSL_CUDA(cudaMemcpyAsync(g->given, host, (size_t)g->n * sizeof(float4), cudaMemcpyHostToDevice, g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_set_body_force(psl_grid* g, float gx, float gy, float gz) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_body_force: null grid");
  g->body = make_float3(gx, gy, gz);
  return PSL_OK;
}

// ---- scalar transport ----
static GridView<StoreF32> scalar_view(const psl_grid* g) {
  GridView<StoreF32> v;
  for (int q = 0; q < 27; ++q) {
    v.fq[q] = g->T + (size_t)q * g->stride;
    v.shift[q] = g->shift[q];
  }
  v.n = g->n;
  return v;
}

int psl_enable_scalar_transport(psl_grid* g, float tauT) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_enable_scalar_transport: null grid");
  PSL_CHECK(tauT > 0.5f, PSL_ERR_INVALID, "psl_enable_scalar_transport: tau_T must exceed 1/2");
  DeviceGuard dg(g->device);
  if (!g->T) {
    const size_t bytes = 27 * g->stride * sizeof(float);
    cudaError_t e = cudaMalloc(&g->T, bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->T, 0, bytes, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) {
      if (g->T) cudaFree(g->T);
      g->T = nullptr;
      cudaGetLastError();
      return fail(PSL_ERR_NOMEM, std::string("psl_enable_scalar_transport: ") + cudaGetErrorString(e));
    }
  }
  g->tauT = tauT;
  return PSL_OK;
}

int psl_set_scalar_given_field(psl_grid* g, const float* host) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_scalar_given_field: null grid");
  DeviceGuard dg(g->device);
  if (!host) {
    if (g->givenT) {
      PSL_CUDA(cudaStreamSynchronize(g->stream));
      cudaFree(g->givenT);
      g->givenT = nullptr;
    }
    return PSL_OK;
  }
  if (!g->givenT) PSL_CUDA(cudaMalloc(&g->givenT, (size_t)g->n * sizeof(float)));
  PSL_CUDA(cudaMemcpyAsync(g->givenT, host, (size_t)g->n * sizeof(float), cudaMemcpyHostToDevice, g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

static int scalar_rows(psl_grid* g, float* host, bool get) {
  float* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * sizeof(float)));
  cudaError_t e = cudaStreamSynchronize(g->stream);
  const GridView<StoreF32> v = scalar_view(g);
  for (int q = 0; q < 27 && e == cudaSuccess; ++q) {
    if (get) {
      gather_logical_kernel<StoreF32><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(v, q, tmp);
      e = cudaGetLastError();
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(host + (size_t)q * g->n, tmp, (size_t)g->n * sizeof(float), cudaMemcpyDeviceToHost, g->stream);
    } else {
      e = cudaMemcpyAsync(tmp, host + (size_t)q * g->n, (size_t)g->n * sizeof(float), cudaMemcpyHostToDevice, g->stream);
      if (e == cudaSuccess) {
        scatter_logical_kernel<StoreF32><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(v, q, tmp);
        e = cudaGetLastError();
      }
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl scalar populations: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_get_scalar_populations(psl_grid* g, float* host) {
  PSL_CHECK(g && host && g->T, PSL_ERR_INVALID, "psl_get_scalar_populations: no scalar transport on this grid");
  DeviceGuard dg(g->device);
  return scalar_rows(g, host, true);
}

int psl_set_scalar_populations(psl_grid* g, const float* host) {
  PSL_CHECK(g && host && g->T, PSL_ERR_INVALID, "psl_set_scalar_populations: no scalar transport on this grid");
  DeviceGuard dg(g->device);
  return scalar_rows(g, const_cast<float*>(host), false);
}

int psl_get_scalar(psl_grid* g, double* host) {
  PSL_CHECK(g && host && g->T, PSL_ERR_INVALID, "psl_get_scalar: no scalar transport on this grid");
  DeviceGuard dg(g->device);
  double* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * sizeof(double)));
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    scalar_mean_kernel<S><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(view<S>(g), scalar_view(g), tmp);
    return 0;
  });
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, (size_t)g->n * sizeof(double), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_get_scalar: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_set_smagorinsky(psl_grid* g, float cs) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_smagorinsky: null grid");
  g->cs = cs;
  return PSL_OK;
}

int psl_set_smagorinsky_field(psl_grid* g, const float* host_cs) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_set_smagorinsky_field: null grid");
  DeviceGuard dg(g->device);
  if (!host_cs) {
    if (g->cs_field) {
      PSL_CUDA(cudaStreamSynchronize(g->stream));
      cudaFree(g->cs_field);
      g->cs_field = nullptr;
    }
    return PSL_OK;
  }
  for (uint32_t c = 0; c < g->n; ++c)
    PSL_CHECK(std::isfinite(host_cs[c]) && host_cs[c] >= 0.f, PSL_ERR_INVALID,
              "psl_set_smagorinsky_field: every constant must be finite and >= 0");
  if (!g->cs_field) {
    cudaError_t e = cudaMalloc(&g->cs_field, g->stride * sizeof(float));
    if (e != cudaSuccess) {
      g->cs_field = nullptr;
      cudaGetLastError();
      return fail(PSL_ERR_NOMEM, std::string("psl_set_smagorinsky_field: ") + cudaGetErrorString(e));
    }
    PSL_CUDA(cudaMemsetAsync(g->cs_field, 0, g->stride * sizeof(float), g->stream));
  }
  PSL_CUDA(cudaMemcpyAsync(g->cs_field, host_cs, (size_t)g->n * sizeof(float), cudaMemcpyHostToDevice, g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

// ---- per-step update ----
template <typename Case>
static int fill_eq(psl_grid* g, const Case& c) {
  DeviceGuard dg(g->device);
  const unsigned int nb = blocks_for(g->n, 256);
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    fill_equilibrium_kernel<S, Case><<<nb, 256, 0, g->stream>>>(view<S>(g), c, hook_info(g));
    return 0;
  });
  PSL_CUDA(cudaGetLastError());
  return PSL_OK;
}

int psl_fill_equilibrium_sphere(psl_grid* g, const psl_sphere_case* sc) {
  PSL_CHECK(g && sc, PSL_ERR_INVALID, "psl_fill_equilibrium_sphere: null argument");
  psl_detail_closure_stale(g);
  return fill_eq(g, sphere_hooks(sc));
}

int psl_fill_equilibrium_uniform(psl_grid* g, float rho, float ux, float uy, float uz) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_fill_equilibrium_uniform: null grid");
  psl_detail_closure_stale(g);
  UniformCase c{rho, ux, uy, uz};
  return fill_eq(g, c);
}

int psl_fill_equilibrium_field(psl_grid* g, const float* rho_u) {
  PSL_CHECK(g && rho_u, PSL_ERR_INVALID, "psl_fill_equilibrium_field: null argument");
  psl_detail_closure_stale(g);
  DeviceGuard dg(g->device);
  float* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * 4 * sizeof(float)));
  cudaError_t e = cudaMemcpyAsync(tmp, rho_u, (size_t)g->n * 4 * sizeof(float), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) {
    with_storage(g->storage, [&](auto s) {
      using S = decltype(s);
      fill_equilibrium_field_kernel<S><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(view<S>(g), tmp);
      return 0;
    });
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_fill_equilibrium_field: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_apply_streaming(psl_grid* g) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_apply_streaming: null grid");
  const long long nx = g->info.cell_count_x, ny = g->info.cell_count_y, n = g->n;
  for (int q = 0; q < 27; ++q) {
    long long s = (long long)g->shift[q];
    s -= cx(q);
    s -= nx * cy(q);
    s -= ny * nx * cz(q);
    if (s < 0) s += n;
    if (s < 0) s += n;
    if (s >= n) s -= n;
    if (s >= n) s -= n;
    g->shift[q] = (uint32_t)s;
  }
  return PSL_OK;
}

// Thread-to-cell rotation of the update kernels (cell_of_thread): half a warp when the x-rows
// are whole warps long, so that each row boundary's two x-face cells share one warp.
uint32_t psl_detail_thread_rotation(const psl_grid* g) {
  return (g->info.cell_count_x % 32 == 0 && g->n > 16) ? 16u : 0u;
}
static uint32_t thread_rotation(const psl_grid* g) { return psl_detail_thread_rotation(g); }

template <typename T>
static RelaxationT<T> relaxation(const psl_grid* g) {
  RelaxationT<T> rx;
  rx.tau = T(3) * T(g->info.nu) + T(0.5);
  rx.tau2 = rx.tau * rx.tau;
  rx.omega0 = T(1) / rx.tau;
  rx.cs18 = T(18) * T(g->cs);
  return rx;
}

// held_nu: the update between two evaluations of the learned closure, on its held nu_t.
template <typename S>
static cudaError_t launch_step(psl_grid* g, bool held_nu, const ThreadRange& range) {
  StepParams<S> p;
  p.g = view<S>(g);
  p.marker = g->marker;
  p.given = g->given;
  p.given_uniform = g->given_uniform;
  p.cs = g->cs_field;
  p.rx = relaxation<typename S::calc>(g);
  p.health = g->health;
  p.ri = row_index<S>(g);
  p.rot = thread_rotation(g);
  p.nut = g->mlp_nut;
  p.nu = g->info.nu;
  p.range = range;
  const unsigned int blocks = blocks_for(range.count, kStepThreads);
  const int addr = 27 * g->f_stride + g->n >= (1ull << 32) ? kAddrView : g->f_twice ? kAddrFlat : kAddrIndex;
  auto launch = [&](auto kernel) { kernel<<<blocks, kStepThreads, 0, g->stream>>>(p); };
  if constexpr (kCollidesOnG<S>) {
    const int rate = held_nu ? kRateNuField : g->cs_field ? kRateCsField : kRateUniform;
    auto pick = [&](auto addr_tag) {
      constexpr int A = decltype(addr_tag)::value;
      if (rate == kRateNuField) launch(step_kernel_g<S, A, kRateNuField>);
      else if (rate == kRateCsField) launch(step_kernel_g<S, A, kRateCsField>);
      else launch(step_kernel_g<S, A, kRateUniform>);
    };
    if (addr == kAddrView) pick(std::integral_constant<int, kAddrView>());
    else if (addr == kAddrFlat) pick(std::integral_constant<int, kAddrFlat>());
    else pick(std::integral_constant<int, kAddrIndex>());
  } else {
    if (addr == kAddrView) launch(step_kernel<S, kAddrView>);
    else if (addr == kAddrFlat) launch(step_kernel<S, kAddrFlat>);
    else launch(step_kernel<S, kAddrIndex>);
  }
  return cudaGetLastError();
}

// The update of the threads in `range` for the plain and the learned-closure paths (the
// closure's network, or its kept nu_t between two runs of it); count_update advances the
// closure's update counter once per update of the whole grid.
static int update_cells(psl_grid* g, const ThreadRange& range) {
  if (g->mlp && !(g->mlp_nut && g->mlp_since != 0)) return psl_detail_launch_learned(g, range);
  const bool held = g->mlp != nullptr;  // between two runs of the closure: its held nu_t
  PSL_CUDA(with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    if constexpr (kCollidesOnG<S>) return launch_step<S>(g, held, range);
    else return held ? cudaErrorInvalidValue : launch_step<S>(g, false, range);  // kept nu_t: 16-bit only
  }));
  return PSL_OK;
}
static void count_update(psl_grid* g) {
  if (g->mlp) g->mlp_since = (g->mlp_since + 1) % g->mlp_interval;
}

int psl_apply_local_cell_update(psl_grid* g) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_apply_local_cell_update: null grid");
  DeviceGuard dg(g->device);
  const bool custom = g->custom_markers || g->body.x != 0.f || g->body.y != 0.f || g->body.z != 0.f;
  if (g->T) {
    PSL_CHECK(!custom && !g->mlp, PSL_ERR_INVALID,
              "psl_apply_local_cell_update: scalar transport does not combine with forcing, moving walls or the "
              "learned closure");
    PSL_CHECK(g->storage != kStoreF64 && 27ull * g->f_stride + g->n < (1ull << 32) && 27ull * g->stride + g->n < (1ull << 32), PSL_ERR_INVALID,
              "psl_apply_local_cell_update: scalar transport needs FP32/FP16/BF16 storage");
    with_storage(g->storage, [&](auto s) {
      using S = decltype(s);
      if constexpr (S::kind != kStoreF64) {
        ScalarParams<S> sp;
        sp.base.g = view<S>(g);
        sp.base.ri = row_index<S>(g);
        sp.base.marker = g->marker;
        sp.base.given = g->given;
        sp.base.given_uniform = g->given_uniform;
        sp.base.cs = g->cs_field;
        sp.base.rx = relaxation<float>(g);
        sp.base.health = g->health;
        sp.T.base = g->T;
        sp.T.n = g->n;
        for (int q = 0; q < 27; ++q) {  // the scalar rows: one plain allocation of row stride `stride`
          sp.T.off[q] = (uint32_t)((size_t)q * g->stride + g->shift[q]);
          sp.T.lim[q] = sp.base.ri.lim[q];
        }
        sp.givenT = g->givenT;
        sp.tauT = g->tauT;
        step_scalar_kernel<S><<<blocks_for(g->n, kStepThreads), kStepThreads, 0, g->stream>>>(sp);
      }
      return 0;
    });
    PSL_CUDA(cudaGetLastError());
    return PSL_OK;
  }
  if (g->mlp) {
    PSL_CHECK(!custom, PSL_ERR_INVALID,
              "psl_apply_local_cell_update: the learned closure does not combine with forcing or moving walls");
    const int rc = update_cells(g, full_range(g->n));
    if (rc == PSL_OK) count_update(g);
    return rc;
  }
  if (custom) {
    PSL_CHECK(g->storage != kStoreF64 && 27ull * g->f_stride + g->n < (1ull << 32), PSL_ERR_INVALID,
              "psl_apply_local_cell_update: forcing and moving walls need FP32/FP16/BF16 storage");
    with_storage(g->storage, [&](auto s) {
      using S = decltype(s);
      if constexpr (S::kind != kStoreF64) {
        CustomParams<S> cp;
        cp.base.g = view<S>(g);
        cp.base.ri = row_index<S>(g);
        cp.base.marker = g->marker;
        cp.base.given = g->given;
        cp.base.given_uniform = g->given_uniform;
        cp.base.cs = g->cs_field;
        cp.base.rx = relaxation<float>(g);
        cp.base.health = g->health;
        cp.body = g->body;
        step_custom_kernel<S><<<blocks_for(g->n, kStepThreads), kStepThreads, 0, g->stream>>>(cp);
      }
      return 0;
    });
    PSL_CUDA(cudaGetLastError());
    return PSL_OK;
  }
  return update_cells(g, full_range(g->n));
}

template <typename S>
static void launch_periodic(psl_grid* g, int axis) {
  const int nx = g->info.cell_count_x, ny = g->info.cell_count_y, nz = g->info.cell_count_z;
  const int items = (axis == 0 ? ny : nx) * nz;
  if (axis == 0)
    periodic_kernel<S, 0><<<blocks_for(items, 256), 256, 0, g->stream>>>(view<S>(g), nx, ny, nz);
  else
    periodic_kernel<S, 1><<<blocks_for(items, 256), 256, 0, g->stream>>>(view<S>(g), nx, ny, nz);
}

static int periodic(psl_grid* g, int axis) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_apply_bc_periodic: null grid");
  DeviceGuard dg(g->device);
  with_storage(g->storage, [&](auto s) {
    launch_periodic<decltype(s)>(g, axis);
    return 0;
  });
  PSL_CUDA(cudaGetLastError());
  return PSL_OK;
}
int psl_apply_bc_periodic_x(psl_grid* g) { return periodic(g, 0); }
int psl_apply_bc_periodic_y(psl_grid* g) { return periodic(g, 1); }

template <typename S>
static int launch_coarse_fine(psl_grid* c, psl_grid* f) {
  const psl_info& C = c->info;
  const psl_info& F = f->info;
  const int a = C.i_subgrid_end - C.i_subgrid_start, b = C.j_subgrid_end - C.j_subgrid_start,
            cc = C.k_subgrid_end - C.k_subgrid_start;
  CoarseFineParams<S> p;
  p.c = row_index<S>(c);
  p.f = row_index<S>(f);
  p.cnx = C.cell_count_x;
  p.cny = C.cell_count_y;
  p.cnz = C.cell_count_z;
  p.iS = C.i_subgrid_start; p.jS = C.j_subgrid_start; p.kS = C.k_subgrid_start;
  p.iE = C.i_subgrid_end; p.jE = C.j_subgrid_end; p.kE = C.k_subgrid_end;
  p.fnx = F.cell_count_x;
  p.fny = F.cell_count_y;
  p.fnz = F.cell_count_z;
  p.fine_marker = f->marker;
  p.face_active = 0;
  if (p.iS > 0) p.face_active |= 1;
  if (p.iE < p.cnx - 1) p.face_active |= 2;
  if (p.jS > 0) p.face_active |= 4;
  if (p.jE < p.cny - 1) p.face_active |= 8;
  if (p.kS > 0) p.face_active |= 16;
  if (p.kE < p.cnz - 1) p.face_active |= 32;
  const long long ra = a - 2, rb = b - 2, rc = cc - 2;
  p.n_ring = (uint32_t)(ra * rb * rc - (ra - 2) * (rb - 2) * (rc - 2));
  // z faces, y faces, then four lanes per x-row boundary (coarse_fine_kernel)
  p.n_shell = (uint32_t)(4LL * p.fnx * p.fny + 4LL * p.fnx * (p.fnz - 4) + 4LL * (p.fny - 3) * (p.fnz - 4));
  const unsigned int ring_blocks = std::max(1u, blocks_for(p.n_ring, kCoarseFineThreads));
  const unsigned int shell_blocks = std::max(1u, blocks_for(p.n_shell, kCoarseFineThreads));
  if (c->f_twice && f->f_twice) {  // both grids' rows mapped twice: no wrap test
    coarse_fine_kernel<S, 1, true><<<ring_blocks, kCoarseFineThreads, 0, c->stream>>>(p);
    coarse_fine_kernel<S, 2, true><<<shell_blocks, kCoarseFineThreads, 0, c->stream>>>(p);
  } else {
    coarse_fine_kernel<S, 1, false><<<ring_blocks, kCoarseFineThreads, 0, c->stream>>>(p);
    coarse_fine_kernel<S, 2, false><<<shell_blocks, kCoarseFineThreads, 0, c->stream>>>(p);
  }
  PSL_CUDA(cudaGetLastError());
  return PSL_OK;
}

// The geometry the restriction reads: both grids' rows, dimensions and the block bounds.
template <typename S>
static CoarseFineParams<S> block_params(psl_grid* c, psl_grid* f) {
  CoarseFineParams<S> p{};
  p.c = row_index<S>(c);
  p.f = row_index<S>(f);
  p.cnx = c->info.cell_count_x;
  p.cny = c->info.cell_count_y;
  p.cnz = c->info.cell_count_z;
  p.iS = c->info.i_subgrid_start; p.jS = c->info.j_subgrid_start; p.kS = c->info.k_subgrid_start;
  p.iE = c->info.i_subgrid_end; p.jE = c->info.j_subgrid_end; p.kE = c->info.k_subgrid_end;
  p.fnx = f->info.cell_count_x;
  p.fny = f->info.cell_count_y;
  p.fnz = f->info.cell_count_z;
  return p;
}

template <typename S>
static int launch_fill_coarse(psl_grid* c, psl_grid* f) {
  const CoarseFineParams<S> p = block_params<S>(c, f);
  const uint32_t cells = (uint32_t)(p.iE - p.iS - 2) * (uint32_t)(p.jE - p.jS - 2) * (uint32_t)(p.kE - p.kS - 2);
  fill_coarse_kernel<S><<<blocks_for(cells, kCoarseFineThreads), kCoarseFineThreads, 0, c->stream>>>(p);
  PSL_CUDA(cudaGetLastError());
  return PSL_OK;
}

int psl_fill_coarse_grid_from_fine(psl_grid* c, psl_grid* f) {
  PSL_CHECK(c && f, PSL_ERR_INVALID, "psl_fill_coarse_grid_from_fine: null grid");
  psl_detail_closure_stale(c);
  PSL_CHECK(c->storage == f->storage, PSL_ERR_INVALID,
            "psl_fill_coarse_grid_from_fine: coarse and fine grids use different storage");
  const psl_info& C = c->info;
  const psl_info& F = f->info;
  const int a = C.i_subgrid_end - C.i_subgrid_start, b = C.j_subgrid_end - C.j_subgrid_start,
            cc = C.k_subgrid_end - C.k_subgrid_start;
  PSL_CHECK(a >= 4 && b >= 4 && cc >= 4, PSL_ERR_INVALID, "fill coarse: refinement block needs >= 4 cells per axis");
  PSL_CHECK(F.cell_count_x == 2 * a && F.cell_count_y == 2 * b && F.cell_count_z == 2 * cc, PSL_ERR_INVALID,
            "fill coarse: fine grid is not twice the refinement block");
  PSL_CHECK(c->device == f->device, PSL_ERR_INVALID, "fill coarse: grids on different devices");
  PSL_CHECK(27ull * c->f_stride + c->n < (1ull << 32) && 27ull * f->f_stride + f->n < (1ull << 32), PSL_ERR_INVALID,
            "fill coarse: grid too large for 32-bit row offsets");
  DeviceGuard dg(c->device);
  return with_storage(c->storage, [&](auto s) { return launch_fill_coarse<decltype(s)>(c, f); });
}

int psl_apply_coarse_fine_grid_communication(psl_grid* c, psl_grid* f) {
  PSL_CHECK(c && f, PSL_ERR_INVALID, "psl_apply_coarse_fine_grid_communication: null grid");
  PSL_CHECK(c->storage == f->storage, PSL_ERR_INVALID,
            "psl_apply_coarse_fine_grid_communication: coarse and fine grids use different storage");
  const psl_info& C = c->info;
  const psl_info& F = f->info;
  const int a = C.i_subgrid_end - C.i_subgrid_start, b = C.j_subgrid_end - C.j_subgrid_start,
            cc = C.k_subgrid_end - C.k_subgrid_start;
  PSL_CHECK(a >= 4 && b >= 4 && cc >= 4, PSL_ERR_INVALID, "coarse/fine: refinement block needs >= 4 cells per axis");
  PSL_CHECK(F.cell_count_x == 2 * a && F.cell_count_y == 2 * b && F.cell_count_z == 2 * cc, PSL_ERR_INVALID,
            "coarse/fine: fine grid is not twice the refinement block");
  PSL_CHECK(c->device == f->device, PSL_ERR_INVALID, "coarse/fine: grids on different devices");
  PSL_CHECK(27ull * c->f_stride + c->n < (1ull << 32) && 27ull * f->f_stride + f->n < (1ull << 32), PSL_ERR_INVALID,
            "coarse/fine: grid too large for 32-bit row offsets");
  DeviceGuard dg(c->device);
  return with_storage(c->storage, [&](auto s) { return launch_coarse_fine<decltype(s)>(c, f); });
}

// psl_update_grid's concurrent schedule for the top coarse grid c of a refined hierarchy.
// The coarse update is split by z-layers into the near slab around the refinement block
// (layers kS - 2 .. kE + 1: every coarse cell the transfer reads or writes lies in layers
// kS - 1 .. kE) and the far layers.  In the PS update each cell reads and writes only its own
// 27 elements (include/applyLocalCellUpdate.h:34,71), so the far cells share no element with
// the transfer and none with the fine grid: the near slab runs first on the grid's stream,
// the far layers then on a lowest-priority side stream beside the two fine updates and the
// transfer (restriction and prolongation: ordinary launches, which can share SMs) on a
// highest-priority stream, and the grid's stream waits for both at the end of the step.  A kernel's launch parameters are fixed
// when it is queued, so the far launch uses this step's shifts wherever it runs.  The result is the serial
// schedule's, bit for bit.  Threads [near.t_begin, near.t_begin + near.count) of
// cell_of_thread cover the near slab; the far launch runs every other thread.
static bool concurrent_fits(psl_grid** grids, int levels, ThreadRange& near, ThreadRange& far) {
  if (levels < 2) return false;
  psl_grid* c = grids[0];
  for (int l = 1; l < levels; ++l)
    if (!grids[l] || grids[l]->stream != c->stream || grids[l]->device != c->device) return false;
  const bool custom = c->custom_markers || c->body.x != 0.f || c->body.y != 0.f || c->body.z != 0.f;
  if (c->T || custom || c->batched) return false;
  const psl_info& I = c->info;
  if (I.i_subgrid_end <= I.i_subgrid_start) return false;
  const long long layer = (long long)I.cell_count_x * I.cell_count_y;
  const long long k0 = I.k_subgrid_start - 2, k1 = (long long)I.k_subgrid_end + 2;  // near: [k0, k1)
  if (k0 < 1 || k1 > I.cell_count_z - 1) return false;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(c->stream, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return false;
  }
  const long long rot = thread_rotation(c), n = c->n;
  const long long A = (k0 * layer + rot) / kStepThreads * kStepThreads;
  const long long B = std::min(n, (k1 * layer + rot + kStepThreads - 1) / kStepThreads * kStepThreads);
  if (!(0 < A && A < B && B < n)) return false;
  near = ThreadRange{(uint32_t)A, 0xffffffffu, 0u, (uint32_t)(B - A)};
  far = ThreadRange{0u, (uint32_t)A, (uint32_t)(B - A), (uint32_t)(n - (B - A))};
  return true;
}

static int concurrent_step(psl_grid** grids, int levels, const ThreadRange& near, const ThreadRange& far) {
  psl_grid* c = grids[0];
  DeviceGuard dg(c->device);
  if (!c->ev_hi) {
    int least = 0, greatest = 0;
    PSL_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    if (!c->side) PSL_CUDA(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, least));
    if (!c->hi) PSL_CUDA(cudaStreamCreateWithPriority(&c->hi, cudaStreamNonBlocking, greatest));
    if (!c->ev_near) PSL_CUDA(cudaEventCreateWithFlags(&c->ev_near, cudaEventDisableTiming));
    if (!c->ev_far) PSL_CUDA(cudaEventCreateWithFlags(&c->ev_far, cudaEventDisableTiming));
    PSL_CUDA(cudaEventCreateWithFlags(&c->ev_hi, cudaEventDisableTiming));
  }
  int rc = psl_apply_streaming(c);
  if (rc) return rc;
  rc = update_cells(c, near);
  if (rc) return rc;
  // Once the near slab is done, the far layers run on the lowest-priority stream and the fine
  // updates and the transfer on the highest-priority one, whatever the priority of the
  // grid's own stream: the block scheduler hands SMs to the fine updates first and the far
  // layers fill in behind them, above all beside the transfer, whose launches alone keep
  // few warps busy.
  PSL_CUDA(cudaEventRecord(c->ev_near, c->stream));
  PSL_CUDA(cudaStreamWaitEvent(c->side, c->ev_near, 0));
  PSL_CUDA(cudaStreamWaitEvent(c->hi, c->ev_near, 0));
  cudaStream_t own = c->stream;
  c->stream = c->side;
  rc = update_cells(c, far);
  c->stream = own;
  if (rc) return rc;
  count_update(c);
  PSL_CUDA(cudaEventRecord(c->ev_far, c->side));
  for (int l = 0; l < levels; ++l) grids[l]->stream = c->hi;
  for (int i = 0; i < 2 && rc == PSL_OK; ++i) rc = psl_update_grid(grids, levels, 1);
  if (rc == PSL_OK) rc = psl_apply_coarse_fine_grid_communication(c, grids[1]);
  for (int l = 0; l < levels; ++l) grids[l]->stream = own;
  // the grid's stream waits for both, also after a failed fine update or transfer
  cudaError_t e = cudaEventRecord(c->ev_hi, c->hi);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(own, c->ev_hi, 0);
  const cudaError_t e_far = cudaStreamWaitEvent(own, c->ev_far, 0);
  if (rc) return rc;
  if (e == cudaSuccess) e = e_far;
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_update_grid: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_update_grid(psl_grid** grids, int levels, int level) {
  PSL_CHECK(grids && levels > 0 && level >= 0 && level < levels, PSL_ERR_INVALID, "psl_update_grid: bad levels");
  ThreadRange near, far;
  if (level == 0 && grids[0] && concurrent_fits(grids, levels, near, far)) return concurrent_step(grids, levels, near, far);
  int rc = psl_apply_streaming(grids[level]);
  if (rc) return rc;
  rc = psl_apply_local_cell_update(grids[level]);
  if (rc) return rc;
  if (level < levels - 1) {
    for (int i = 0; i < 2; ++i) {
      rc = psl_update_grid(grids, levels, level + 1);
      if (rc) return rc;
    }
    rc = psl_apply_coarse_fine_grid_communication(grids[level], grids[level + 1]);
    if (rc) return rc;
  }
  return PSL_OK;
}

// ---- reductions ----
template <typename S>
static void launch_force(psl_grid* g, int i0, int j0, int k0, int si, int sj, int sk, int nb) {
  force_partial_kernel<S><<<nb, 256, 0, g->stream>>>(view<S>(g), g->marker, g->info.cell_count_x,
                                                     g->info.cell_count_y, i0, j0, k0, si, sj, sk, g->scratch);
}

// Enqueues the momentum-exchange force of the sphere's box on the grid's stream; the
// result (3 doubles) lands in `force3` (device or pinned host memory) when the stream
// reaches the copy.  Returns 1 with nothing enqueued when the box is empty.
static int enqueue_sphere_force(psl_grid* g, const psl_sphere_case* sc, double* force3, cudaMemcpyKind kind) {
  const psl_info& I = g->info;
  // bounding box as getSphereDrag computes it (flowAroundSphereMainSingle.cu:105-110)
  int i0 = (int)((sc->sphere_x - sc->sphere_r - I.ox) / I.res);
  int i1 = (int)((sc->sphere_x + sc->sphere_r - I.ox) / I.res) + 2;
  int j0 = (int)((sc->sphere_y - sc->sphere_r - I.oy) / I.res);
  int j1 = (int)((sc->sphere_y + sc->sphere_r - I.oy) / I.res) + 2;
  int k0 = (int)((sc->sphere_z - sc->sphere_r - I.oz) / I.res);
  int k1 = (int)((sc->sphere_z + sc->sphere_r - I.oz) / I.res) + 2;
  i0 = std::max(i0, 0); j0 = std::max(j0, 0); k0 = std::max(k0, 0);
  i1 = std::min(i1, I.cell_count_x); j1 = std::min(j1, I.cell_count_y); k1 = std::min(k1, I.cell_count_z);
  if (i1 <= i0 || j1 <= j0 || k1 <= k0) return 1;
  const int si = i1 - i0, sj = j1 - j0, sk = k1 - k0;
  const int nb = (int)std::min<long long>(kForceBlocks, ((long long)si * sj * sk + 255) / 256);
  with_storage(g->storage, [&](auto s) {
    launch_force<decltype(s)>(g, i0, j0, k0, si, sj, sk, nb);
    return 0;
  });
  force_final_kernel<<<1, 256, 0, g->stream>>>(g->scratch, nb, g->scratch + kForceBlocks * 3);
  PSL_CUDA(cudaGetLastError());
  PSL_CUDA(cudaMemcpyAsync(force3, g->scratch + kForceBlocks * 3, 3 * sizeof(double), kind, g->stream));
  return PSL_OK;
}

int psl_sphere_force(psl_grid* g, const psl_sphere_case* sc, double* force3) {
  PSL_CHECK(g && sc && force3, PSL_ERR_INVALID, "psl_sphere_force: null argument");
  DeviceGuard dg(g->device);
  force3[0] = force3[1] = force3[2] = 0.0;
  const int rc = enqueue_sphere_force(g, sc, force3, cudaMemcpyDeviceToHost);
  if (rc == 1) return PSL_OK;
  if (rc != PSL_OK) return rc;
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_sphere_force_async(psl_grid* g, const psl_sphere_case* sc, double* force3) {
  PSL_CHECK(g && sc && force3, PSL_ERR_INVALID, "psl_sphere_force_async: null argument");
  DeviceGuard dg(g->device);
  const int rc = enqueue_sphere_force(g, sc, force3, cudaMemcpyDefault);
  if (rc == 1) {  // empty box: zeros, in stream order like the non-empty case
    PSL_CUDA(cudaMemsetAsync(g->scratch + kForceBlocks * 3, 0, 3 * sizeof(double), g->stream));
    PSL_CUDA(cudaMemcpyAsync(force3, g->scratch + kForceBlocks * 3, 3 * sizeof(double), cudaMemcpyDefault, g->stream));
    return PSL_OK;
  }
  return rc;
}

// ---- data movement ----
// FP32 storage needs no conversion: logical row q is the stored row rotated by shift_q
// (cell c at (c + shift_q) mod N), so it moves with plain copies -- one contiguous range on
// twice-mapped rows (the second mapping holds the wrap), else the two pieces of the
// rotation -- without a staging buffer or a kernel.
static cudaError_t copy_rows_f32(psl_grid* g, float* host, bool to_host) {
  float* base = static_cast<float*>(g->f);
  const size_t n = g->n;
  for (int q = 0; q < 27; ++q) {
    float* row = base + (size_t)q * g->f_stride;
    float* h = host + (size_t)q * n;
    const size_t sh = g->shift[q];
    const size_t first = g->f_twice ? n : n - sh;  // elements of the first piece
    cudaError_t e = to_host ? cudaMemcpyAsync(h, row + sh, first * sizeof(float), cudaMemcpyDeviceToHost, g->stream)
                            : cudaMemcpyAsync(row + sh, h, first * sizeof(float), cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess && first < n)
      e = to_host ? cudaMemcpyAsync(h + first, row, (n - first) * sizeof(float), cudaMemcpyDeviceToHost, g->stream)
                  : cudaMemcpyAsync(row, h + first, (n - first) * sizeof(float), cudaMemcpyHostToDevice, g->stream);
    if (e != cudaSuccess) return e;
  }
  return cudaStreamSynchronize(g->stream);
}

template <typename S>
static int gather(psl_grid* g, float* host) {
  if constexpr (S::kind == kStoreF32) {
    const cudaError_t e = copy_rows_f32(g, host, true);
    if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_get_populations: ") + cudaGetErrorString(e));
    return PSL_OK;
  }
  float* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * sizeof(float)));
  cudaError_t e = cudaSuccess;
  const GridView<S> v = view<S>(g);
  // one staging row; stream order serialises each row's gather after the previous copy
  for (int q = 0; q < 27 && e == cudaSuccess; ++q) {
    gather_logical_kernel<S><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(v, q, tmp);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(host + (size_t)q * g->n, tmp, (size_t)g->n * sizeof(float), cudaMemcpyDeviceToHost, g->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_get_populations: ") + cudaGetErrorString(e));
  return PSL_OK;
}

template <typename S>
static int scatter(psl_grid* g, const float* host) {
  if constexpr (S::kind == kStoreF32) {
    const cudaError_t e = copy_rows_f32(g, const_cast<float*>(host), false);
    if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_set_populations: ") + cudaGetErrorString(e));
    return PSL_OK;
  }
  float* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * sizeof(float)));
  cudaError_t e = cudaSuccess;
  const GridView<S> v = view<S>(g);
  for (int q = 0; q < 27 && e == cudaSuccess; ++q) {
    e = cudaMemcpyAsync(tmp, host + (size_t)q * g->n, (size_t)g->n * sizeof(float), cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess) {
      scatter_logical_kernel<S><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(v, q, tmp);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_set_populations: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_get_populations(psl_grid* g, float* host) {
  PSL_CHECK(g && host, PSL_ERR_INVALID, "psl_get_populations: null argument");
  DeviceGuard dg(g->device);
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return with_storage(g->storage, [&](auto s) { return gather<decltype(s)>(g, host); });
}

int psl_get_macroscopic(psl_grid* g, double* host) {
  PSL_CHECK(g && host, PSL_ERR_INVALID, "psl_get_macroscopic: null argument");
  DeviceGuard dg(g->device);
  double* tmp = nullptr;
  PSL_CUDA(cudaMalloc(&tmp, (size_t)g->n * 4 * sizeof(double)));
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    macroscopic_kernel<S><<<blocks_for(g->n, 256), 256, 0, g->stream>>>(view<S>(g), tmp);
    return 0;
  });
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, tmp, (size_t)g->n * 4 * sizeof(double), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_get_macroscopic: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_set_populations(psl_grid* g, const float* host) {
  PSL_CHECK(g && host, PSL_ERR_INVALID, "psl_set_populations: null argument");
  psl_detail_closure_stale(g);
  DeviceGuard dg(g->device);
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return with_storage(g->storage, [&](auto s) { return scatter<decltype(s)>(g, host); });
}

int psl_get_shifts(const psl_grid* g, int* s) {
  PSL_CHECK(g && s, PSL_ERR_INVALID, "psl_get_shifts: null argument");
  for (int q = 0; q < 27; ++q) s[q] = (int)g->shift[q];
  return PSL_OK;
}

int psl_set_shifts(psl_grid* g, const int* s) {
  PSL_CHECK(g && s, PSL_ERR_INVALID, "psl_set_shifts: null argument");
  psl_detail_closure_stale(g);
  for (int q = 0; q < 27; ++q)
    PSL_CHECK(s[q] >= 0 && (uint32_t)s[q] < g->n, PSL_ERR_INVALID, "psl_set_shifts: shift outside [0, N)");
  for (int q = 0; q < 27; ++q) g->shift[q] = (uint32_t)s[q];
  return PSL_OK;
}

int psl_synchronize(psl_grid* g) {
  PSL_CHECK(g, PSL_ERR_INVALID, "psl_synchronize: null grid");
  DeviceGuard dg(g->device);
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_check_health(psl_grid* g, unsigned int* flags) {
  PSL_CHECK(g && flags, PSL_ERR_INVALID, "psl_check_health: null argument");
  DeviceGuard dg(g->device);
  PSL_CUDA(cudaMemcpyAsync(flags, g->health, sizeof(unsigned int), cudaMemcpyDeviceToHost, g->stream));
  PSL_CUDA(cudaMemsetAsync(g->health, 0, sizeof(unsigned int), g->stream));
  PSL_CUDA(cudaStreamSynchronize(g->stream));
  return PSL_OK;
}

int psl_debug_cells(int op, int a0, float* host_f, const float* host_args, int count) {
  PSL_CHECK(host_f && host_args && count > 0, PSL_ERR_INVALID, "psl_debug_cells: bad argument");
  int ndev = 0;
  PSL_CUDA(cudaGetDeviceCount(&ndev));
  PSL_CHECK(ndev > 0, PSL_ERR_CUDA, "psl_debug_cells: no CUDA device");
  float *df = nullptr, *da = nullptr;
  PSL_CUDA(cudaMalloc(&df, (size_t)count * 27 * sizeof(float)));
  cudaError_t e = cudaMalloc(&da, (size_t)count * 4 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(df, host_f, (size_t)count * 27 * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(da, host_args, (size_t)count * 4 * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    debug_cell_kernel<<<blocks_for(count, 64), 64>>>(op, a0, df, da, count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(host_f, df, (size_t)count * 27 * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(df);
  if (da) cudaFree(da);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_debug_cells: ") + cudaGetErrorString(e));
  return PSL_OK;
}

