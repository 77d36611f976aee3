// Full-grid right side of the reference's Krylov path (BuildRhs2D,
// src/backends/cpu/solver.cpp:167-232: Dirichlet values on boundary rows,
// -f inside) and the one-shot operator apply behind pdeb200_apply
// (LinearOperator2D::Apply, src/backends/cpu/cpu_utils.cpp:324-513).
#include "host.h"
#include "solvers.cuh"

namespace pdeb {

__global__ void k_full_rhs(GridDev g, const double* __restrict__ f, double f_const, double* __restrict__ b) {
  for (long long t = gtid(); t < g.n; t += gstride()) {
    const int i = int(t % g.nx);
    const int j = int((t / g.nx) % g.ny);
    const int k = int(t / g.sxy);
    const bool on[6] = {i == 0, i == g.nx - 1, j == 0, j == g.ny - 1, g.dim == 3 && k == 0,
                        g.dim == 3 && k == g.nz - 1};
    const bool bd = on[0] || on[1] || on[2] || on[3] || on[4] || on[5];
    if (!bd) {
      b[t] = -(f ? f[t] : f_const);
      continue;
    }
    double v = 0.0;
    for (int q = 5; q >= 0; --q)
      if (on[q] && g.face[q].active && g.face[q].kind == kDirichlet) {
        v = g.face[q].val.at(face_loc(g, q, i, j, k));
        break;
      }
    b[t] = v;
  }
}

pdeb200_status apply_dev(Context* ctx, DevProblem& P, const double* d_x, double* d_y) {
  with_coef(P, [&](const auto& cf) {
    using Coef = std::decay_t<decltype(cf)>;
    k_apply_full<Coef, 0, NoPost><<<stencil_grid_full(P.g), stencil_block(), 0, ctx->stream>>>(
        P.g, cf, d_x, d_y, RedSlot{}, NoPost{}, nullptr);
  });
  ctx->count();
  return PDEB200_OK;
}

}  // namespace pdeb
