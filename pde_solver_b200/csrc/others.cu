// Drivers not yet specialised for the B200 path report UNSUPPORTED.
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

template <class Coef>
pdeb200_status gauss_seidel(Context*, DevProblem&, const Coef&, const pdeb200_options*, double*, pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "Gauss-Seidel/SOR not built yet"};
}
template <class Coef>
pdeb200_status bicgstab_reference(Context*, DevProblem&, const Coef&, const pdeb200_options*, double*,
                                  pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "BiCGStab not built yet"};
}
template <class Coef>
pdeb200_status gmres_reference(Context*, DevProblem&, const Coef&, const pdeb200_options*, double*, pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "GMRES not built yet"};
}
pdeb200_status mg_vcycle_reference(Context*, DevProblem&, const pdeb200_problem*, const pdeb200_options*, double*,
                                   pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "reference V-cycle not built yet"};
}
template <class Coef>
pdeb200_status mixed_refinement(Context*, DevProblem&, const Coef&, const pdeb200_problem*, const pdeb200_options*,
                                double*, pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "mixed precision not built yet"};
}
template <class Coef>
pdeb200_status mg_bicgstab(Context*, DevProblem&, const Coef&, const pdeb200_problem*, const pdeb200_options*,
                           double*, pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "MG-BiCGStab not built yet"};
}

#define INST(C)                                                                                                   \
  template pdeb200_status gauss_seidel<C>(Context*, DevProblem&, const C&, const pdeb200_options*, double*,       \
                                          pdeb200_report*);                                                       \
  template pdeb200_status bicgstab_reference<C>(Context*, DevProblem&, const C&, const pdeb200_options*, double*, \
                                                pdeb200_report*);                                                 \
  template pdeb200_status gmres_reference<C>(Context*, DevProblem&, const C&, const pdeb200_options*, double*,    \
                                             pdeb200_report*);                                                    \
  template pdeb200_status mixed_refinement<C>(Context*, DevProblem&, const C&, const pdeb200_problem*,            \
                                              const pdeb200_options*, double*, pdeb200_report*);                  \
  template pdeb200_status mg_bicgstab<C>(Context*, DevProblem&, const C&, const pdeb200_problem*,                 \
                                         const pdeb200_options*, double*, pdeb200_report*);
INST(CoefConst)
INST(CoefDivk<double>)
INST(CoefNodal)

pdeb200_status residual_norms_dev(Context*, DevProblem&, const double*, double*, double*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "residual norms not built yet"};
}
pdeb200_status time_series_dev(Context*, DevProblem&, const pdeb200_time_options*, pdeb200_frame_cb, void*, bool,
                               double*, pdeb200_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "time series not built yet"};
}
pdeb200_status project_dev(Context*, int, int, int, double, double, double, double, double*, double*, double*,
                           double*, const pdeb200_projection_options*, pdeb200_projection_report*) {
  throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "projection not built yet"};
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
