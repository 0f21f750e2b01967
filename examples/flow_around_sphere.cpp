// A reference-style case driver on the C++ mirror (include/psl.hpp): the loop of
// flowAroundSphere/flowAroundSphereMainSingle.cu:245-264 -- updateGrid, then the drag --
// on the 512x256x256 sphere case with one 2:1 refinement level.
//
//   g++ -O2 -std=c++17 -I include examples/flow_around_sphere.cpp \
//       periodicshiftlbm_b200/libpsl_b200.so -Wl,-rpath,$PWD/periodicshiftlbm_b200 -o sphere
//   ./sphere [steps]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "psl.hpp"

int main(int argc, char** argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 100;
  psl_sphere_case sc{};
  sc.sphere_x = sc.sphere_y = sc.sphere_z = 128.f;
  sc.sphere_r = 24.f;
  sc.u_in = 0.05f;
  sc.rho_given = 1.f;
  sc.wall_mode = 0;
  sc.smagorinsky = 0.1f;
  sc.seed = 1234;
  sc.noise_amp = 1e-4f;

  std::vector<psl::GridStruct> grids(2);
  psl::InfoStruct c;
  c.cellCountX = 512;
  c.cellCountY = c.cellCountZ = 256;
  c.nu = 0.05f * 48.f / 1e5f;
  c.iSubgridStart = c.jSubgridStart = c.kSubgridStart = 80;
  c.iSubgridEnd = 208;
  c.jSubgridEnd = c.kSubgridEnd = 176;
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
  const auto t0 = std::chrono::steady_clock::now();
  double drag = 0.0;
  for (int it = 0; it < steps; ++it) {
    psl::updateGrid(grids, 0);
    drag = psl::getSphereDrag(grids[1], sc);
  }
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const double updates = 512.0 * 256 * 256 - 124.0 * 92 * 92 + 2.0 * 254 * 190 * 190;
  std::printf("steps %d  drag %.6g  MLUPS %.1f (with a drag read-back every step)\n", steps, drag,
              updates * steps / s / 1e6);
  return 0;
}
