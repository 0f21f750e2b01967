// Host build of the 16-bit forms' collision on g = f - w (psl_collision_g.cuh) for the
// CPU tests: count cells of 27 deviations each, collided in place.
#include "psl_collision_g.cuh"

extern "C" void collide_g_host(float* g, int count, float nu, float cs) {
  const float tau = 3.f * nu + 0.5f;
  for (int c = 0; c < count; ++c) {
    float v[27];
    for (int q = 0; q < 27; ++q) v[q] = g[27 * c + q];
    const psl::CellMomentsG m = psl::cell_moments_g(v);
    const float w = psl::smagorinsky_omega_g(m, 1.f / tau, tau, tau * tau, 18.f * cs);
    psl::relax_rebuild_g(v, m, w);
    for (int q = 0; q < 27; ++q) g[27 * c + q] = v[q];
  }
}
