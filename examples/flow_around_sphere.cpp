// A reference-style case driver on the C++ mirror (include/psl.hpp): the loop of
// flowAroundSphere/flowAroundSphereMainSingle.cu:245-264 -- updateGrid, then the drag --
// on the 512x256x256 sphere case with one 2:1 refinement level (every length times
// `scale`, the Reynolds number kept, as periodicshiftlbm_b200.cases.config2(scale)).
//
//   g++ -O2 -std=c++17 -I include examples/flow_around_sphere.cpp
//       periodicshiftlbm_b200/libpsl_b200.so -Wl,-rpath,$PWD/periodicshiftlbm_b200 -o sphere
//   (one command line)
//   ./sphere [steps] [scale] [sponge]
// With "sponge" the coarse grid takes a per-cell getSmagorinskyConstant hook: C_s rising
// linearly from the case's constant at i = 3 Nx / 4 to four times it at the outlet
// (periodicshiftlbm_b200.cases.sponge_smagorinsky is the same hook in Python).
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "psl.hpp"

int main(int argc, char** argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 100;
  const double scale = argc > 2 ? std::atof(argv[2]) : 1.0;
  const bool sponge = argc > 3 && std::string(argv[3]) == "sponge";
  auto sc_len = [&](double v) { return (int)std::lround(v * scale); };
  psl_sphere_case sc{};
  sc.sphere_x = sc.sphere_y = sc.sphere_z = (float)(128.0 * scale);
  sc.sphere_r = (float)(24.0 * scale);
  sc.u_in = 0.05f;
  sc.rho_given = 1.f;
  sc.wall_mode = 0;
  sc.smagorinsky = 0.1f;
  sc.seed = 1234;
  sc.noise_amp = 1e-4f;

  std::vector<psl::GridStruct> grids(2);
  psl::InfoStruct c;
  c.cellCountX = sc_len(512);
  c.cellCountY = c.cellCountZ = sc_len(256);
  c.nu = (float)(0.05 * 48 * scale / 1e5);
  c.iSubgridStart = c.jSubgridStart = c.kSubgridStart = sc_len(80);
  c.iSubgridEnd = sc_len(208);
  c.jSubgridEnd = c.kSubgridEnd = sc_len(176);
  psl::InfoStruct f;  // flowAroundSphereMainSingle.cu:185-215
  f.gridID = 1;
  f.res = c.res * 0.5f;
  f.dtPhys = c.dtPhys * 0.5f;
  f.nu = c.nu * 2.f;
  f.ox = c.ox + c.iSubgridStart * c.res - f.res * 0.5f;
  f.oy = c.oy + c.jSubgridStart * c.res - f.res * 0.5f;
  f.oz = c.oz + c.kSubgridStart * c.res - f.res * 0.5f;
  f.cellCountX = (c.iSubgridEnd - c.iSubgridStart) * 2;
  f.cellCountY = (c.jSubgridEnd - c.jSubgridStart) * 2;
  f.cellCountZ = (c.kSubgridEnd - c.kSubgridStart) * 2;
  grids[0].create(c);
  grids[1].create(f);
  for (auto& g : grids) {
    psl::setSphereCase(g, sc);
    psl::fillEquilibriumFromFunction(g, sc);
  }
  if (sponge) {
    const float cs = sc.smagorinsky;
    psl::setSmagorinskyConstant(grids[0], [cs](int i, int, int, const psl::InfoStruct& I) {
      const int i0 = (3 * I.cellCountX) / 4;
      float ramp = 3.f * (float)(i - i0);
      ramp = ramp / (float)(I.cellCountX - 1 - i0);
      return i > i0 ? cs * (1.f + ramp) : cs;
    });
  }
  const auto t0 = std::chrono::steady_clock::now();
  double drag = 0.0;
  for (int it = 0; it < steps; ++it) {
    psl::updateGrid(grids, 0);
    drag = psl::getSphereDrag(grids[1], sc);
  }
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  // cells updated per coarse step: the coarse grid less its refined interior, twice the
  // fine grid less its ghost layer (include/applyLocalCellUpdate.h:25-30)
  const double updates = (double)c.cellCountX * c.cellCountY * c.cellCountZ -
                         (double)(c.iSubgridEnd - c.iSubgridStart - 4) * (c.jSubgridEnd - c.jSubgridStart - 4) *
                             (c.kSubgridEnd - c.kSubgridStart - 4) +
                         2.0 * (f.cellCountX - 2) * (f.cellCountY - 2) * (f.cellCountZ - 2);
  std::printf("steps %d  drag %.17g  MLUPS %.1f (with a drag read-back every step)\n", steps, drag,
              updates * steps / s / 1e6);
  return 0;
}
