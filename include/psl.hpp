// psl.hpp -- header-only C++ mirror of the reference's per-step API over the C ABI (psl.h).
//
// A reference case file (flowAroundSphere/flowAroundSphereMainSingle.cu) calls
//   applyStreaming(Grid); applyLocalCellUpdate(Grid); applyCoarseFineGridCommunication(C, F);
//   fillEquilibriumFromFunction(Grid); getSphereDrag(Grid) ...
// on TNL-backed GridStruct objects.  Including this header instead gives the same calls on
// GridStruct objects whose state lives on the B200 and whose update runs in the
// project's sm_100a kernels.  Errors throw psl::Error (the reference's TNL containers
// throw on CUDA failures too); the C ABI underneath never throws.
#pragma once

#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "psl.h"

namespace psl {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& what) : std::runtime_error(what), code(c) {}
};

inline void check(int rc, const char* what) {
  if (rc != PSL_OK) throw Error(rc, std::string(what) + ": " + psl_last_error());
}

// InfoStruct (include/types.h:73-75) with the reference's field names.
struct InfoStruct {
  float gridID = 0;
  float res = 1.f;
  int cellCountX = 0, cellCountY = 0, cellCountZ = 0, cellCount = 0;
  float ox = 0.f, oy = 0.f, oz = 0.f;
  float nu = 1.f;
  float dtPhys = 1.f;
  int iSubgridStart = 0, jSubgridStart = 0, kSubgridStart = 0;
  int iSubgridEnd = 0, jSubgridEnd = 0, kSubgridEnd = 0;

  psl_info to_c() const {
    psl_info i{};
    i.grid_id = (int)gridID;
    i.res = res;
    i.cell_count_x = cellCountX;
    i.cell_count_y = cellCountY;
    i.cell_count_z = cellCountZ;
    i.ox = ox;
    i.oy = oy;
    i.oz = oz;
    i.nu = nu;
    i.dt_phys = dtPhys;
    i.i_subgrid_start = iSubgridStart;
    i.j_subgrid_start = jSubgridStart;
    i.k_subgrid_start = kSubgridStart;
    i.i_subgrid_end = iSubgridEnd;
    i.j_subgrid_end = jSubgridEnd;
    i.k_subgrid_end = kSubgridEnd;
    return i;
  }
};

// GridStruct (include/types.h:77): owns one device grid.
class GridStruct {
 public:
  InfoStruct Info;

  GridStruct() = default;
  explicit GridStruct(const InfoStruct& info, int storage = PSL_STORAGE_F32) { create(info, storage); }
  GridStruct(const GridStruct&) = delete;
  GridStruct& operator=(const GridStruct&) = delete;
  GridStruct(GridStruct&& o) noexcept : Info(o.Info), h_(std::exchange(o.h_, nullptr)) {}
  GridStruct& operator=(GridStruct&& o) noexcept {
    if (this != &o) {
      reset();
      Info = o.Info;
      h_ = std::exchange(o.h_, nullptr);
    }
    return *this;
  }
  ~GridStruct() { reset(); }

  void create(const InfoStruct& info, int storage = PSL_STORAGE_F32) {
    reset();
    Info = info;
    Info.cellCount = info.cellCountX * info.cellCountY * info.cellCountZ;
    const psl_info c = Info.to_c();
    check(psl_grid_create(&c, storage, &h_), "psl_grid_create");
  }
  void reset() {
    if (h_) psl_grid_destroy(h_);
    h_ = nullptr;
  }
  psl_grid* handle() const { return h_; }

  // fArray in logical order, [27][cellCount]
  std::vector<float> populations() const {
    std::vector<float> f((size_t)27 * Info.cellCount);
    check(psl_get_populations(h_, f.data()), "psl_get_populations");
    return f;
  }
  void setPopulations(const std::vector<float>& f) { check(psl_set_populations(h_, f.data()), "psl_set_populations"); }
  std::vector<int> shifter() const {
    std::vector<int> s(27);
    check(psl_get_shifts(h_, s.data()), "psl_get_shifts");
    return s;
  }

 private:
  psl_grid* h_ = nullptr;
};

// ---- the reference's free functions ----
inline void applyStreaming(GridStruct& g) { check(psl_apply_streaming(g.handle()), "applyStreaming"); }
inline void applyLocalCellUpdate(GridStruct& g) {
  check(psl_apply_local_cell_update(g.handle()), "applyLocalCellUpdate");
}
inline void applyBCPeriodicX(GridStruct& g) { check(psl_apply_bc_periodic_x(g.handle()), "applyBCPeriodicX"); }
inline void applyBCPeriodicY(GridStruct& g) { check(psl_apply_bc_periodic_y(g.handle()), "applyBCPeriodicY"); }
inline void applyCoarseFineGridCommunication(GridStruct& coarse, GridStruct& fine) {
  check(psl_apply_coarse_fine_grid_communication(coarse.handle(), fine.handle()), "applyCoarseFineGridCommunication");
}
inline void fillCoarseGridFromFine(GridStruct& coarse, GridStruct& fine) {
  check(psl_fill_coarse_grid_from_fine(coarse.handle(), fine.handle()), "fillCoarseGridFromFine");
}
// fillEquilibriumFromFunction with the sphere case's start hook, or a uniform state.
inline void fillEquilibriumFromFunction(GridStruct& g, const psl_sphere_case& sc) {
  check(psl_fill_equilibrium_sphere(g.handle(), &sc), "fillEquilibriumFromFunction");
}
inline void fillEquilibriumUniform(GridStruct& g, float rho, float ux, float uy, float uz) {
  check(psl_fill_equilibrium_uniform(g.handle(), rho, ux, uy, uz), "fillEquilibriumUniform");
}
// getMarkers / getGivenRhoUxUyUz / getSmagorinskyConstant of the sphere case.
inline void setSphereCase(GridStruct& g, const psl_sphere_case& sc) {
  check(psl_apply_sphere_case(g.handle(), &sc), "setSphereCase");
}
// A case's getSmagorinskyConstant(i, j, k, Info) hook (include/applyLocalCellUpdate.h:68),
// any callable with that signature returning the constant: evaluated once per cell on the
// host, in cell order, and kept on the device as the grid's per-cell field.
template <typename Hook>
inline void setSmagorinskyConstant(GridStruct& g, Hook&& getSmagorinskyConstant) {
  const InfoStruct& I = g.Info;
  std::vector<float> cs((size_t)I.cellCountX * I.cellCountY * I.cellCountZ);
  size_t c = 0;
  for (int k = 0; k < I.cellCountZ; ++k)
    for (int j = 0; j < I.cellCountY; ++j)
      for (int i = 0; i < I.cellCountX; ++i) cs[c++] = (float)getSmagorinskyConstant(i, j, k, I);
  check(psl_set_smagorinsky_field(g.handle(), cs.data()), "setSmagorinskyConstant");
}
// The uniform form (one constant for every cell; 0 disables LES).
inline void setSmagorinskyConstant(GridStruct& g, float cs) {
  check(psl_set_smagorinsky(g.handle(), cs), "setSmagorinskyConstant");
}
// The customised update (moving walls, forced-velocity cells, body force): see
// psl_set_body_force in psl.h for the marker bytes.
inline void setBodyForce(GridStruct& g, float gx, float gy, float gz) {
  check(psl_set_body_force(g.handle(), gx, gy, gz), "setBodyForce");
}
inline void getTorque(GridStruct& g, const int lo[3], const int hi[3], const float point[3], double torque[3],
                      double force[3]) {
  check(psl_torque(g.handle(), lo, hi, point, torque, force), "getTorque");
}

// updateGrid recursion of the case driver (flowAroundSphereMainSingle.cu:158-167).
inline void updateGrid(std::vector<GridStruct>& grids, int level) {
  std::vector<psl_grid*> h(grids.size());
  for (size_t i = 0; i < grids.size(); ++i) h[i] = grids[i].handle();
  check(psl_update_grid(h.data(), (int)h.size(), level), "updateGrid");
}
// getSphereDrag in lattice units of `g` (FP64), before convertToPhysicalForce.
inline double getSphereDrag(GridStruct& g, const psl_sphere_case& sc) {
  double f[3];
  check(psl_sphere_force(g.handle(), &sc, f), "getSphereDrag");
  return f[0];
}
// The same force queued without a host wait: `force3` (device or pinned host memory) holds
// it once the grid's stream has passed this call (synchronize()).
inline void getSphereForceAsync(GridStruct& g, const psl_sphere_case& sc, double* force3) {
  check(psl_sphere_force_async(g.handle(), &sc, force3), "getSphereForceAsync");
}
inline void synchronize(GridStruct& g) { check(psl_synchronize(g.handle()), "synchronize"); }

}  // namespace psl
