// Host build of the generated CUDA boundary-condition header (test harness only).
// Compiled with g++ (no FMA contraction on x86-64), the generated code's explicit
// operation order must reproduce the reference's host results bit for bit.
#include "psl_bc_generated.cuh"

extern "C" void bc_host(int op, int normal, float* f, const float* a) {
  float (&v)[27] = *reinterpret_cast<float (*)[27]>(f);
  float rho = a[0], ux = a[1], uy = a[2], uz = a[3];
  switch (op) {
    case 2: psl::bc::mbbc(normal, v, rho, ux, uy, uz); break;
    case 3: psl::bc::restore_rho(normal, v, rho, ux, uy, uz); v[0] = rho; break;
    case 4: psl::bc::restore_u(normal, v, rho, ux, uy, uz); v[0] = ux; v[1] = uy; v[2] = uz; break;
    case 5: psl::bc::restore_rho_u(normal, v, rho, ux, uy, uz); v[0] = rho; v[1] = ux; v[2] = uy; v[3] = uz; break;
    case 6: psl::bc::mirror(normal, v); break;
    default: break;
  }
}
