// Flow reports (include/psl.h): torque of the momentum exchange on solid cells and the
// plane flow report composed over refinement levels (FP64 reductions), and the section-cut
// export of the reference's plotters.
//
// psl_get_flow_report follows getFlowReportGeneral (include/flowReportFunctions.h:2-251): the
// physical bounds are mapped to index bounds on the finest grid; the finest level whose
// cropped section has fewer than 20,000,000 pixels is the target resolution; every level,
// coarsest first, paints the cells that intersect the cut plane into the section (a
// coarser cell covers cellScale/targetScale pixels per direction, finer levels overwrite
// coarser ones); pixels of solid cells are excluded; the report is the mean velocity,
// 1 + mean(rho - 1) and the area (pixel count x target cell size^2).  The sums are FP64
// here (the reference reduces in FP32).  Levels are placed by their origins (ox, oy, oz),
// so a refined PS grid lands where it lies in the coarse grid.
//
// psl_forcing_torque is the reference's getTorque (M35Full/m35Main.cu:176-260) on PS grids:
// -g_x y + g_y x summed over the forced-velocity cells, g their forcing in physical units.
// psl_torque sums r x F over the solid cells of a box, F the per-cell momentum exchange of
// getSphereDrag (flowAroundSphereMainSingle.cu:99-156, rho (u - u_bounced)) and r the cell
// centre minus a reference point: the same moment for bounce-back bodies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "psl.h"
#include "psl_internal.h"
#include "psl_kernels.cuh"

using namespace psl;

namespace {

int fail(int code, const std::string& msg) {
  psl_detail_set_last_error(msg);
  return code;
}

#define REP_CUDA(expr)                                                                                 \
  do {                                                                                                 \
    cudaError_t e_ = (expr);                                                                           \
    if (e_ != cudaSuccess) return fail(PSL_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename Fn>
auto with_storage(int storage, Fn&& fn) {
  switch (storage) {
    case kStoreF32: return fn(StoreF32{});
    case kStoreF16: return fn(StoreF16{});
    case kStoreBF16: return fn(StoreBF16{});
    default: return fn(StoreF64{});
  }
}

template <typename S>
GridView<S> view_of(const psl_grid* g) {
  GridView<S> v;
  typename S::type* base = static_cast<typename S::type*>(g->f);
  for (int q = 0; q < 27; ++q) {
    v.fq[q] = base + (size_t)q * g->f_stride;
    v.shift[q] = g->shift[q];
  }
  v.n = g->n;
  return v;
}

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 256;

// Block sums of `nv` FP64 values per item, written per block; final kernel sums in order.
template <int NV>
__device__ __forceinline__ void block_sum_store(double (&v)[NV], double* partial) {
  __shared__ double red[NV][kRedThreads];
  for (int c = 0; c < NV; ++c) red[c][threadIdx.x] = v[c];
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int c = 0; c < NV; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int c = 0; c < NV; ++c) partial[blockIdx.x * NV + c] = red[c][0];
}

template <int NV>
__global__ void final_sum_kernel(const double* partial, int blocks, double* out) {
  const int c = threadIdx.x;
  if (c >= NV) return;
  double s = 0.0;
  for (int b = 0; b < blocks; ++b) s += partial[b * NV + c];
  out[c] = s;
}

// torque (3) and force (3) of the solid cells of [i0,i0+si) x [j0,j0+sj) x [k0,k0+sk)
template <typename S>
__global__ void __launch_bounds__(kRedThreads) torque_kernel(GridView<S> g, const uint8_t* marker, int nx, int ny,
                                                             int i0, int j0, int k0, int si, int sj, int sk, float res,
                                                             float ox, float oy, float oz, float px, float py, float pz,
                                                             double* partial) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const uint32_t total = (uint32_t)si * sj * sk;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int i = i0 + (int)(t % si), j = j0 + (int)((t / si) % sj), k = k0 + (int)(t / (si * sj));
    const uint32_t cell = ((uint32_t)k * ny + j) * nx + i;
    if (marker_kind(marker[cell]) != kSolid) continue;
    double jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      const double v = (double)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
      jx += cx(q) * v;
      jy += cy(q) * v;
      jz += cz(q) * v;
    }
    // rho (u - u_bounced) = 2 j (the bounced populations carry -j)
    const double fx = 2.0 * jx, fy = 2.0 * jy, fz = 2.0 * jz;
    const double rx = (double)i * res + ox - px, ry = (double)j * res + oy - py, rz = (double)k * res + oz - pz;
    acc[0] += ry * fz - rz * fy;
    acc[1] += rz * fx - rx * fz;
    acc[2] += rx * fy - ry * fx;
    acc[3] += fx;
    acc[4] += fy;
    acc[5] += fz;
  }
  block_sum_store<6>(acc, partial);
}

// getTorque (M35Full/m35Main.cu:176-260) on a PS grid: per forced-velocity cell with
// k >= k_min, the forcing g = rho (u_given - u) of its stored populations (the target of
// the library's forced cells is their given velocity, where the reference's getForcing hook
// computes one), in physical units (convertToPhysicalForce, cellFunctions.h:221-226:
// times rho_nominal (res/1000)^4 / dt^2), and its torque -g_x y + g_y x about the z axis
// through the origin, (x, y) = (i res + ox, j res + oy) as getXYZFromIJKCellIndex gives
// them.  Sums: torque, g (physical) -- four FP64 values.
template <typename S>
__global__ void __launch_bounds__(kRedThreads) forcing_torque_kernel(GridView<S> g, const uint8_t* marker,
                                                                     const float4* given, float4 given_uniform, int nx,
                                                                     int ny, int k_min, float res, float ox, float oy,
                                                                     double to_phys, double* partial) {
  double acc[4] = {0, 0, 0, 0};
  for (uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.n; cell += gridDim.x * blockDim.x) {
    const uint8_t m = marker[cell];
    if (marker_kind(m) != kFluid || marker_normal(m) != 1) continue;  // forced-velocity cells
    const int k = (int)(cell / ((uint32_t)nx * ny));
    if (k < k_min) continue;
    const uint32_t r = cell - (uint32_t)k * nx * ny;
    const int j = (int)(r / nx), i = (int)(r % nx);
    double rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
      const double v = (double)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
      rho += v;
      jx += cx(q) * v;
      jy += cy(q) * v;
      jz += cz(q) * v;
    }
    const float4 gv = given ? given[cell] : given_uniform;
    const double gx = (rho * (double)gv.y - jx) * to_phys;
    const double gy = (rho * (double)gv.z - jy) * to_phys;
    const double gz = (rho * (double)gv.w - jz) * to_phys;
    const float x = (float)i * res + ox, y = (float)j * res + oy;
    acc[0] += -gx * (double)y + gy * (double)x;
    acc[1] += gx;
    acc[2] += gy;
    acc[3] += gz;
  }
  block_sum_store<4>(acc, partial);
}

struct Section {
  float* rho;
  float* ux;
  float* uy;
  float* uz;
  uint8_t* solid;
  int width, height;
};

// Paint the cells of one level that intersect the cut into the section.  (a, b) index the
// level's in-plane cells (horizontal, vertical axes of the plane), `layer` its cut layer.
template <typename S>
__global__ void section_kernel(GridView<S> g, const uint8_t* marker, int nx, int ny, int plane, int layer, int na,
                               int nb, int scale, int target_scale, int off_h, int off_v, int h_min, int v_min,
                               Section sec) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na * nb) return;
  const int a = t % na, b = t / na;
  int i, j, k;
  if (plane == PSL_PLANE_XY) {
    i = a; j = b; k = layer;
  } else if (plane == PSL_PLANE_ZY) {
    k = a; j = b; i = layer;
  } else {
    k = a; i = b; j = layer;
  }
  const uint32_t cell = ((uint32_t)k * ny + j) * nx + i;
  double rho = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    const double v = (double)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
    rho += v;
    jx += cx(q) * v;
    jy += cy(q) * v;
    jz += cz(q) * v;
  }
  const uint8_t solid = marker_solid(marker[cell]);
  const int h0 = (off_h + a * scale) / target_scale - h_min;
  const int v0 = (off_v + b * scale) / target_scale - v_min;
  const int span = max(1, scale / target_scale);
  for (int dv = 0; dv < span; ++dv) {
    const int y = v0 + dv;
    if (y < 0 || y >= sec.height) continue;
    for (int dh = 0; dh < span; ++dh) {
      const int x = h0 + dh;
      if (x < 0 || x >= sec.width) continue;
      const size_t p = (size_t)y * sec.width + x;
      sec.rho[p] = (float)rho;
      sec.ux[p] = (float)(jx / rho);
      sec.uy[p] = (float)(jy / rho);
      sec.uz[p] = (float)(jz / rho);
      sec.solid[p] = solid;
    }
  }
}

__global__ void __launch_bounds__(kRedThreads) section_sum_kernel(Section sec, double* partial) {
  double acc[5] = {0, 0, 0, 0, 0};  // count, ux, uy, uz, rho - 1
  const size_t total = (size_t)sec.width * sec.height;
  for (size_t p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    if (sec.solid[p]) continue;
    acc[0] += 1.0;
    acc[1] += sec.ux[p];
    acc[2] += sec.uy[p];
    acc[3] += sec.uz[p];
    acc[4] += (double)sec.rho[p] - 1.0;
  }
  block_sum_store<5>(acc, partial);
}

// getRhoUxUyUz (cellFunctions.h:135-155) in FP32 with the reference's order of additions.
__device__ __forceinline__ void rho_u_reference_order(const float (&f)[27], float& rho, float& ux, float& uy, float& uz) {
  float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    r = __fadd_rn(r, f[q]);
    if (cx(q) != 0) jx = cx(q) > 0 ? __fadd_rn(jx, f[q]) : __fsub_rn(jx, f[q]);
    if (cy(q) != 0) jy = cy(q) > 0 ? __fadd_rn(jy, f[q]) : __fsub_rn(jy, f[q]);
    if (cz(q) != 0) jz = cz(q) > 0 ? __fadd_rn(jz, f[q]) : __fsub_rn(jz, f[q]);
  }
  rho = r;
  ux = __fdiv_rn(jx, r);
  uy = __fdiv_rn(jy, r);
  uz = __fdiv_rn(jz, r);
}

// One pixel of exportSectionCutPlotGeneral (include/plotter/exportSectionCutPlot.h:1-88):
// (p, u_horizontal, u_vertical, u_normal, solid) in physical units.
template <typename S>
__global__ void section_export_kernel(GridView<S> g, const uint8_t* marker, int nx, int ny, int plane, int cut,
                                      int horizontal, int vertical, float vel_scale, float dt, float p_scale,
                                      float* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= horizontal * vertical) return;
  const int h = t % horizontal, v = t / horizontal;
  int i, j, k;
  if (plane == PSL_PLANE_XY) {
    i = h; j = v; k = cut;
  } else if (plane == PSL_PLANE_ZY) {
    i = cut; j = v; k = h;
  } else {
    i = v; j = cut; k = h;
  }
  const uint32_t cell = ((uint32_t)k * ny + j) * nx + i;
  float f[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = (float)S::load_q(g.fq[q] + shifted(cell, g.shift[q], g.n), q);
  float rho, ux, uy, uz;
  rho_u_reference_order(f, rho, ux, uy, uz);
  // convertToPhysicalVelocity / convertToPhysicalPressure (cellFunctions.h:200-219)
  ux = __fdiv_rn(__fmul_rn(ux, vel_scale), dt);
  uy = __fdiv_rn(__fmul_rn(uy, vel_scale), dt);
  uz = __fdiv_rn(__fmul_rn(uz, vel_scale), dt);
  const float p = __fmul_rn(__fsub_rn(rho, 1.f), p_scale);
  float uh, uv, un;
  if (plane == PSL_PLANE_XY) {
    uh = ux; uv = uy; un = uz;
  } else if (plane == PSL_PLANE_ZY) {
    uh = uz; uv = uy; un = ux;
  } else {
    uh = uz; uv = ux; un = uy;
  }
  float* o = out + ((size_t)v * horizontal + h) * 5;
  o[0] = p;
  o[1] = uh;
  o[2] = uv;
  o[3] = un;
  o[4] = marker_solid(marker[cell]) ? 1.f : 0.f;
}

}  // namespace

int psl_export_section_cut(psl_grid* g, int plane, int cut, float rho_nominal_phys, float soundspeed_phys,
                           float* out, long long capacity, int* vertical, int* horizontal) {
  if (!g || !vertical || !horizontal || plane < PSL_PLANE_XY || plane > PSL_PLANE_ZX)
    return fail(PSL_ERR_INVALID, "psl_export_section_cut: bad argument");
  const psl_info& I = g->info;
  int H, V, depth;
  if (plane == PSL_PLANE_XY) {
    H = I.cell_count_x; V = I.cell_count_y; depth = I.cell_count_z;
  } else if (plane == PSL_PLANE_ZY) {
    H = I.cell_count_z; V = I.cell_count_y; depth = I.cell_count_x;
  } else {
    H = I.cell_count_z; V = I.cell_count_x; depth = I.cell_count_y;
  }
  *vertical = V;
  *horizontal = H;
  if (!out) return PSL_OK;  // size query
  if (cut < 0 || cut >= depth) return fail(PSL_ERR_INVALID, "psl_export_section_cut: cut index outside the grid");
  const size_t count = (size_t)V * H * 5;
  if (capacity < (long long)count) return fail(PSL_ERR_INVALID, "psl_export_section_cut: output buffer too small");
  DeviceGuard dg(g->device);
  float* dev = nullptr;
  REP_CUDA(cudaMalloc(&dev, count * sizeof(float)));
  // convertToPhysicalVelocity: u (res / 1000) / dtPhys; convertToPhysicalPressure:
  // (rho - 1) rhoNominalPhys soundspeedPhys^2
  const float vel_scale = I.res / 1000.f;
  const float p_scale = rho_nominal_phys * soundspeed_phys * soundspeed_phys;
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    section_export_kernel<S><<<(H * V + 255) / 256, 256, 0, g->stream>>>(view_of<S>(g), g->marker, I.cell_count_x,
                                                                        I.cell_count_y, plane, cut, H, V, vel_scale,
                                                                        I.dt_phys, p_scale, dev);
    return 0;
  });
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dev, count * sizeof(float), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_export_section_cut: ") + cudaGetErrorString(e));
  return PSL_OK;
}

int psl_torque(psl_grid* g, const int* lo3, const int* hi3, const float* point3, double* torque3, double* force3) {
  if (!g || !lo3 || !hi3 || !point3 || !torque3) return fail(PSL_ERR_INVALID, "psl_torque: null argument");
  const psl_info& I = g->info;
  const int i0 = std::max(lo3[0], 0), j0 = std::max(lo3[1], 0), k0 = std::max(lo3[2], 0);
  const int i1 = std::min(hi3[0], I.cell_count_x), j1 = std::min(hi3[1], I.cell_count_y),
            k1 = std::min(hi3[2], I.cell_count_z);
  for (int c = 0; c < 3; ++c) {
    torque3[c] = 0.0;
    if (force3) force3[c] = 0.0;
  }
  if (i1 <= i0 || j1 <= j0 || k1 <= k0) return PSL_OK;
  DeviceGuard dg(g->device);
  double* buf = nullptr;
  REP_CUDA(cudaMalloc(&buf, (kRedBlocks * 6 + 6) * sizeof(double)));
  const long long cells = (long long)(i1 - i0) * (j1 - j0) * (k1 - k0);
  const int nb = (int)std::min<long long>(kRedBlocks, (cells + kRedThreads - 1) / kRedThreads);
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    torque_kernel<S><<<nb, kRedThreads, 0, g->stream>>>(view_of<S>(g), g->marker, I.cell_count_x, I.cell_count_y, i0,
                                                       j0, k0, i1 - i0, j1 - j0, k1 - k0, I.res, I.ox, I.oy, I.oz,
                                                       point3[0], point3[1], point3[2], buf);
    return 0;
  });
  final_sum_kernel<6><<<1, 32, 0, g->stream>>>(buf, nb, buf + kRedBlocks * 6);
  double out[6];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf + kRedBlocks * 6, sizeof(out), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_torque: ") + cudaGetErrorString(e));
  for (int c = 0; c < 3; ++c) {
    torque3[c] = out[c];
    if (force3) force3[c] = out[3 + c];
  }
  return PSL_OK;
}

int psl_forcing_torque(psl_grid* g, int k_min, float rho_nominal_phys, double* torque, double* force3) {
  if (!g || !torque) return fail(PSL_ERR_INVALID, "psl_forcing_torque: null argument");
  const psl_info& I = g->info;
  DeviceGuard dg(g->device);
  double* buf = nullptr;
  REP_CUDA(cudaMalloc(&buf, (kRedBlocks * 4 + 4) * sizeof(double)));
  const int nb = (int)std::min<long long>(kRedBlocks, ((long long)g->n + kRedThreads - 1) / kRedThreads);
  const double len = (double)I.res / 1000.0;
  const double to_phys = (double)rho_nominal_phys * len * len * len * len / ((double)I.dt_phys * I.dt_phys);
  with_storage(g->storage, [&](auto s) {
    using S = decltype(s);
    forcing_torque_kernel<S><<<nb, kRedThreads, 0, g->stream>>>(view_of<S>(g), g->marker, g->given, g->given_uniform,
                                                               I.cell_count_x, I.cell_count_y, k_min, I.res, I.ox,
                                                               I.oy, to_phys, buf);
    return 0;
  });
  final_sum_kernel<4><<<1, 32, 0, g->stream>>>(buf, nb, buf + kRedBlocks * 4);
  double out[4];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf + kRedBlocks * 4, sizeof(out), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_forcing_torque: ") + cudaGetErrorString(e));
  *torque = out[0] / 1000.0;  // N mm -> N m, as the reference reports it
  if (force3)
    for (int c = 0; c < 3; ++c) force3[c] = out[1 + c];
  return PSL_OK;
}

int psl_get_flow_report(psl_grid* const* grids, int levels, int plane, int cut_index, const float* bounds6,
                    psl_flow_report* report) {
  if (!grids || levels < 1 || !bounds6 || !report || plane < PSL_PLANE_XY || plane > PSL_PLANE_ZX)
    return fail(PSL_ERR_INVALID, "psl_get_flow_report: bad argument");
  for (int l = 0; l < levels; ++l)
    if (!grids[l]) return fail(PSL_ERR_INVALID, "psl_get_flow_report: null grid");
  const psl_info& F = grids[levels - 1]->info;  // finest
  auto idx = [&](float v, float o, bool up) { return (int)(up ? std::ceil((v - o) / F.res) : std::floor((v - o) / F.res)); };
  const int iMin = std::max(0, idx(bounds6[0], F.ox, false)), iMax = std::min(F.cell_count_x, idx(bounds6[3], F.ox, true));
  const int jMin = std::max(0, idx(bounds6[1], F.oy, false)), jMax = std::min(F.cell_count_y, idx(bounds6[4], F.oy, true));
  const int kMin = std::max(0, idx(bounds6[2], F.oz, false)), kMax = std::min(F.cell_count_z, idx(bounds6[5], F.oz, true));
  int hMinF, hMaxF, vMinF, vMaxF;
  if (plane == PSL_PLANE_XY) {
    hMinF = iMin; hMaxF = iMax; vMinF = jMin; vMaxF = jMax;
  } else if (plane == PSL_PLANE_ZY) {
    hMinF = kMin; hMaxF = kMax; vMinF = jMin; vMaxF = jMax;
  } else {
    hMinF = kMin; hMaxF = kMax; vMinF = iMin; vMaxF = iMax;
  }
  // the finest level whose cropped section stays under 20,000,000 pixels
  int target_levels = levels, target_scale = 1, W = 0, H = 0, hMin = 0, vMin = 0;
  while (target_levels > 0) {
    target_scale = 1 << (levels - target_levels);
    hMin = hMinF / target_scale;
    vMin = vMinF / target_scale;
    W = std::max(0, (hMaxF + target_scale - 1) / target_scale - hMin);
    H = std::max(0, (vMaxF + target_scale - 1) / target_scale - vMin);
    if ((long long)W * H < 20000000LL || target_levels == 1) break;
    --target_levels;
  }
  report->ux = report->uy = report->uz = 0.0;
  report->rho = 1.0;
  report->area = 0.0;
  if (W == 0 || H == 0) return PSL_OK;
  DeviceGuard dg(grids[0]->device);
  const size_t px = (size_t)W * H;
  Section sec{nullptr, nullptr, nullptr, nullptr, nullptr, W, H};
  double* buf = nullptr;
  cudaError_t e = cudaMalloc(&sec.rho, px * 4 * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&sec.solid, px);
  if (e == cudaSuccess) e = cudaMalloc(&buf, (kRedBlocks * 5 + 5) * sizeof(double));
  if (e != cudaSuccess) {
    cudaFree(sec.rho);
    cudaFree(sec.solid);
    cudaGetLastError();
    return fail(PSL_ERR_NOMEM, std::string("psl_get_flow_report: ") + cudaGetErrorString(e));
  }
  sec.ux = sec.rho + px;
  sec.uy = sec.rho + 2 * px;
  sec.uz = sec.rho + 3 * px;
  cudaStream_t st = grids[levels - 1]->stream;
  for (int l = 0; l < levels; ++l) cudaStreamSynchronize(grids[l]->stream);
  // empty pixels: rho 1, u 0, marked (the reference fills the marker with 1)
  std::vector<float> init(px * 4, 0.f);
  std::fill(init.begin(), init.begin() + px, 1.f);
  e = cudaMemcpyAsync(sec.rho, init.data(), px * 4 * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(sec.solid, 1, px, st);
  const float resF = F.res;
  for (int l = 0; l < levels && e == cudaSuccess; ++l) {
    const psl_grid* g = grids[l];
    const psl_info& I = g->info;
    const int scale = 1 << (levels - 1 - l);
    // origin of this level in finest-cell units
    const int oi = (int)std::lround((I.ox - F.ox) / resF), oj = (int)std::lround((I.oy - F.oy) / resF),
              ok = (int)std::lround((I.oz - F.oz) / resF);
    int layer, na, nb, off_h, off_v, off_c;
    if (plane == PSL_PLANE_XY) {
      off_c = ok; na = I.cell_count_x; nb = I.cell_count_y; off_h = oi; off_v = oj;
    } else if (plane == PSL_PLANE_ZY) {
      off_c = oi; na = I.cell_count_z; nb = I.cell_count_y; off_h = ok; off_v = oj;
    } else {
      off_c = oj; na = I.cell_count_z; nb = I.cell_count_x; off_h = ok; off_v = oi;
    }
    const int rel = cut_index - off_c;
    if (rel < 0) continue;
    layer = rel / scale;
    const int depth = plane == PSL_PLANE_XY ? I.cell_count_z : (plane == PSL_PLANE_ZY ? I.cell_count_x : I.cell_count_y);
    if (layer >= depth) continue;
    with_storage(g->storage, [&](auto s) {
      using S = decltype(s);
      section_kernel<S><<<(na * nb + 255) / 256, 256, 0, st>>>(view_of<S>(g), g->marker, I.cell_count_x, I.cell_count_y,
                                                               plane, layer, na, nb, scale, target_scale, off_h, off_v,
                                                               hMin, vMin, sec);
      return 0;
    });
    e = cudaGetLastError();
  }
  const int nbk = (int)std::min<size_t>(kRedBlocks, (px + kRedThreads - 1) / kRedThreads);
  if (e == cudaSuccess) {
    section_sum_kernel<<<nbk, kRedThreads, 0, st>>>(sec, buf);
    final_sum_kernel<5><<<1, 32, 0, st>>>(buf, nbk, buf + kRedBlocks * 5);
    e = cudaGetLastError();
  }
  double out[5] = {0, 0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, buf + kRedBlocks * 5, sizeof(out), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(sec.rho);
  cudaFree(sec.solid);
  cudaFree(buf);
  if (e != cudaSuccess) return fail(PSL_ERR_CUDA, std::string("psl_get_flow_report: ") + cudaGetErrorString(e));
  if (out[0] > 0) {
    const double res_t = grids[target_levels - 1]->info.res;
    report->area = out[0] * res_t * res_t;
    report->ux = out[1] / out[0];
    report->uy = out[2] / out[0];
    report->uz = out[3] / out[0];
    report->rho = out[4] / out[0] + 1.0;
  }
  return PSL_OK;
}
