// Solver drivers of libpdeb200: the reference methods with the reference's
// semantics (Jacobi, lexicographic GS/SOR, CG, BiCGStab, GMRES, single
// V-cycle "mg") and the B200 forms (MG-preconditioned CG / BiCGStab on the
// folded system, FP32-inside-FP64 refinement). Every iteration runs on the
// device: Krylov scalars are derived by the last block of each fused
// reduction and convergence is decided on the device (Ctl), so the host only
// enqueues and polls.
#include <cmath>
#include <cstring>

#include "host.h"
#include "solvers.cuh"

namespace pdeb {

// ---------------------------------------------------------- relaxation

// Jacobi with the reference sequence (relaxation.cpp:310-574 / solver.cpp:749-981):
// initial closures, then per iteration: sweep grid -> next, closures on next, swap.
template <class Coef>
pdeb200_status jacobi(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_out,
                      pdeb200_report* rep) {
  const GridDev& g = P.g;
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  Buf other(sizeof(double) * g.n, ctx->stream);
  Buf degen(sizeof(int), ctx->stream);
  PDEB_CUDA(cudaMemsetAsync(degen.as<int>(), 0, sizeof(int), ctx->stream));
  double* buf[2] = {d_out, other.as<double>()};
  PDEB_CUDA(cudaMemsetAsync(buf[0], 0, sizeof(double) * g.n, ctx->stream));
  PDEB_CUDA(cudaMemsetAsync(buf[1], 0, sizeof(double) * g.n, ctx->stream));
  ctl_init(ctx, max_iter, o->tol, 0.0);
  fill_boundary(ctx, g, buf[0], ctx->d_ctl);
  const dim3 grid = stencil_grid(g), block = stencil_block();
  auto iterate = [&](int t) {
    double* src = buf[t & 1];
    double* dst = buf[(t + 1) & 1];
    k_jacobi<Coef, PostDelta><<<grid, block, 0, ctx->stream>>>(g, cf, P.f, P.f_const, P.nl, src, dst, ctx->slot(),
                                                               PostDelta{ctx->d_ctl}, ctx->d_ctl, degen.as<int>());
    fill_boundary(ctx, g, dst, ctx->d_ctl);
    ctx->count();
  };
  // kJacobiGroup sweeps (an even number, so each group starts from buf[0])
  // captured once as a CUDA graph and replayed: small grids are launch-bound
  // (129^2: about 11 us per sweep as two direct launches). Sweeps after the
  // stopping test fired return at once, so a group may end past it.
  constexpr int kJacobiGroup = 8;
  auto group = [&](int) {
    for (int t = 0; t < kJacobiGroup; ++t) iterate(t);
  };
  IterGraph graph;
  const bool graphed = graph.capture(ctx, group);
  auto step = [&](int q) {
    if (graphed)
      graph.launch(ctx);
    else
      group(q);
  };
  pdeb200_status st = drive(ctx, o, (max_iter + kJacobiGroup - 1) / kJacobiGroup, step, true);
  const Ctl c = ctl_poll(ctx);
  int dg = 0;
  PDEB_CUDA(cudaMemcpy(&dg, degen.as<int>(), sizeof(int), cudaMemcpyDeviceToHost));
  if (dg) return PDEB200_ERR_DEGENERATE;
  // the converged field is in buf[iter & 1]
  if (c.iter & 1)
    PDEB_CUDA(cudaMemcpyAsync(d_out, buf[1], sizeof(double) * g.n, cudaMemcpyDeviceToDevice, ctx->stream));
  if (rep) {
    rep->iterations = c.iter;
    rep->last_delta = c.delta;
    rep->converged = st == PDEB200_OK;
  }
  return st;
}

// --------------------------------------------------------- reference CG

// CgSolve (krylov.cpp:14-80) on the full grid with identity boundary rows.
template <class Coef>
pdeb200_status cg_reference(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_x,
                            pdeb200_report* rep) {
  const GridDev& g = P.g;
  const long long n = g.n;
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  Buf bb(sizeof(double) * n, ctx->stream), rb(sizeof(double) * n, ctx->stream), pb(sizeof(double) * n, ctx->stream),
      qb(sizeof(double) * n, ctx->stream);
  double *b = bb.as<double>(), *r = rb.as<double>(), *p = pb.as<double>(), *q = qb.as<double>();
  ctl_init(ctx, max_iter, o->tol, 1e-30);
  build_full_rhs(ctx, P, b);
  PDEB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, ctx->stream));
  // x0 = 0 => r = b - A*0 = b
  PDEB_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  const bool relative = o->tol_mode == PDEB200_TOL_RELATIVE;
  const int nb = vec_blocks(n, ctx);
  if (relative) {
    k_dot<double, PostBB><<<nb, 256, 0, ctx->stream>>>(n, b, b, ctx->slot(), PostBB{ctx->d_ctl}, ctx->d_ctl);
    k_dot<double, PostRZ><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostRZ{ctx->d_ctl}, ctx->d_ctl);
  } else {
    k_dot<double, PostRR0Ref><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostRR0Ref{ctx->d_ctl}, ctx->d_ctl);
  }
  ctx->count(relative ? 2 : 1);
  const dim3 grid = stencil_grid_full(g), block = stencil_block();
  auto iterate = [&](int) {
    k_apply_full<Coef, 1, PostAlpha><<<grid, block, 0, ctx->stream>>>(g, cf, p, q, ctx->slot(), PostAlpha{ctx->d_ctl},
                                                                       ctx->d_ctl);
    if (relative) {
      k_cg_xr<double, PostRRRel><<<nb, 256, 0, ctx->stream>>>(n, d_x, r, p, q, ctx->slot(), PostRRRel{ctx->d_ctl},
                                                              ctx->d_ctl);
      k_dot<double, PostBeta><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostBeta{ctx->d_ctl}, ctx->d_ctl);
      ctx->count();
    } else {
      k_cg_xr<double, PostRRRefCG><<<nb, 256, 0, ctx->stream>>>(n, d_x, r, p, q, ctx->slot(),
                                                                PostRRRefCG{ctx->d_ctl}, ctx->d_ctl);
    }
    k_cg_p<double><<<nb, 256, 0, ctx->stream>>>(n, p, r, ctx->d_ctl, 0);
    ctx->count(3);
  };
  pdeb200_status st = drive(ctx, o, max_iter + 1, iterate, false);
  const Ctl c = ctl_poll(ctx);
  if (rep) {
    rep->iterations = c.iter;
    rep->converged = st == PDEB200_OK;
  }
  // true residual of the full system
  full_residual_report(ctx, P, cf, b, d_x, r, rep);
  return st;
}

// ------------------------------------------------------------- MG-PCG

template <class Coef>
pdeb200_status mg_pcg(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_problem* hp,
                      const pdeb200_options* o, double* d_x, pdeb200_report* rep) {
  const GridDev& g = P.g;
  const long long n = g.n;
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  Hierarchy<Coef, double> H;
  H.build(ctx, P, hp, cf, o);
  Buf rb(sizeof(double) * n, ctx->stream), pb(sizeof(double) * n, ctx->stream), qb(sizeof(double) * n, ctx->stream);
  double *r = rb.as<double>(), *p = pb.as<double>(), *q = qb.as<double>();
  double* b = H.levels[0].b;  // level-0 rhs buffer doubles as the folded b
  Buf bsave(sizeof(double) * n, ctx->stream);
  double* bf = bsave.as<double>();
  ctl_init(ctx, max_iter, o->tol, 1e-300);
  build_folded_rhs(ctx, P, cf, bf);
  PDEB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(r, bf, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  PDEB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * n, ctx->stream));
  PDEB_CUDA(cudaMemsetAsync(q, 0, sizeof(double) * n, ctx->stream));
  const int nb = vec_blocks(n, ctx);
  k_dot<double, PostBB><<<nb, 256, 0, ctx->stream>>>(n, bf, bf, ctx->slot(), PostBB{ctx->d_ctl}, ctx->d_ctl);
  ctx->count();
  (void)b;
  // z = M r (z is the level-0 result buffer), p = z, rz = r.z
  double* z = H.z();
  H.vcycle(ctx, r, ctx->d_ctl);
  k_dot<double, PostRZ><<<nb, 256, 0, ctx->stream>>>(n, r, z, ctx->slot(), PostRZ{ctx->d_ctl}, ctx->d_ctl);
  k_cg_p<double><<<nb, 256, 0, ctx->stream>>>(n, p, z, ctx->d_ctl, 1);
  ctx->count(2);
  const dim3 grid = stencil_grid_auto(g), block = stencil_block();
  const double dofs = interior_dofs(g);
  auto iterate = [&](int) {
    {
      ProfScope ps(ctx, "apply_dot", 0, dofs * 24.0);
      launch_dep(ctx, grid, block, 0, k_apply_folded<Coef, double, 1, PostAlpha>, g, cf, (const double*)p, q,
                 ctx->slot(), PostAlpha{ctx->d_ctl}, (const Ctl*)ctx->d_ctl);
    }
    {
      ProfScope ps(ctx, "cg_update_xr", 0, dofs * 48.0);
      launch_dep(ctx, dim3(nb), dim3(256), 0, k_cg_xr<double, PostRRRel>, n, d_x, r, (const double*)p,
                 (const double*)q, ctx->slot(), PostRRRel{ctx->d_ctl}, ctx->d_ctl);
    }
    ctx->count(2);
    // beta from r.z: summed by the preconditioner's last two colour passes
    // when it can, else by a separate dot
    if (!H.vcycle_dot(ctx, r, ctx->d_ctl, ctx->slot())) {
      ProfScope ps(ctx, "dot", 0, dofs * 16.0);
      launch_dep(ctx, dim3(nb), dim3(256), 0, k_dot<double, PostBeta>, n, (const double*)r, (const double*)z,
                 ctx->slot(), PostBeta{ctx->d_ctl}, (const Ctl*)ctx->d_ctl);
    }
    {
      ProfScope ps(ctx, "cg_update_p", 0, dofs * 24.0);
      launch_dep(ctx, dim3(nb), dim3(256), 0, k_cg_p<double>, n, p, (const double*)z, (const Ctl*)ctx->d_ctl, 0);
    }
    ctx->count(2);
  };
  IterGraph graph;
  const bool graphed = graph.capture(ctx, iterate);
  auto step = [&](int it) {
    if (graphed)
      graph.launch(ctx);
    else
      iterate(it);
  };
  // |r|^2 <= tol2 on the device (PostRRRel): batches sized by the observed reduction rate
  pdeb200_status st = drive(ctx, o, max_iter + 1, step, false, true);
  const Ctl c = ctl_poll(ctx);
  if (rep) {
    rep->iterations = c.iter;
    rep->converged = st == PDEB200_OK;
    rep->rhs_l2 = std::sqrt(c.bb);
  }
  folded_residual_report(ctx, P, cf, bf, d_x, r, rep);
  fill_boundary(ctx, g, d_x, nullptr);
  return st;
}

// --------------------------------------------------------------- dispatch

pdeb200_status solve_dispatch(Context* ctx, DevProblem& P, const pdeb200_problem* hp, const pdeb200_options* o,
                              double* d_out, pdeb200_report* rep) {
  if (o->max_iter < 0 || !(o->tol >= 0.0)) throw StatusFailure{PDEB200_ERR_INVALID, "invalid iteration limits"};
  PDEB_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
  pdeb200_status st = PDEB200_ERR_UNSUPPORTED;
  const bool all_dirichlet = [&] {
    for (int f = 0; f < 6; ++f)
      if (P.g.face[f].active && P.g.face[f].kind != kDirichlet) return false;
    return true;
  }();
  const bool relaxation = o->method == PDEB200_JACOBI || o->method == PDEB200_GAUSS_SEIDEL || o->method == PDEB200_SOR;
  if (P.coef_kind == kConst && std::fabs(P.cc.c) < 1e-12 && relaxation)
    throw StatusFailure{PDEB200_ERR_DEGENERATE, "degenerate PDE center coefficient"};
  // pointwise nonlinear terms: relaxation only (src/backends/cpu/solver.cpp:502,550)
  if (P.nl.n > 0 && !relaxation)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, o->method == PDEB200_CG || o->method == PDEB200_BICGSTAB ||
                                                         o->method == PDEB200_GMRES
                                                     ? "Krylov solvers require linear PDEs"
                                                     : "Multigrid requires linear PDEs"};
  with_coef(P, [&](const auto& cf) {
    switch (o->method) {
      case PDEB200_JACOBI:
        st = jacobi(ctx, P, cf, o, d_out, rep);
        break;
      case PDEB200_GAUSS_SEIDEL:
      case PDEB200_SOR:
        st = gauss_seidel(ctx, P, cf, o, d_out, rep);
        break;
      case PDEB200_CG:
      case PDEB200_BICGSTAB:
      case PDEB200_GMRES:
        if (!all_dirichlet)
          throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "Krylov solvers require Dirichlet boundaries on all sides"};
        if (o->method == PDEB200_CG)
          st = cg_reference(ctx, P, cf, o, d_out, rep);
        else if (o->method == PDEB200_BICGSTAB)
          st = bicgstab_reference(ctx, P, cf, o, d_out, rep);
        else
          st = gmres_reference(ctx, P, cf, o, d_out, rep);
        break;
      case PDEB200_MG_VCYCLE:
        st = mg_vcycle_reference(ctx, P, hp, o, d_out, rep);
        break;
      case PDEB200_MG_PCG:
        if (o->precision == PDEB200_MIXED)
          st = mixed_refinement(ctx, P, cf, hp, o, d_out, rep);
        else
          st = mg_pcg(ctx, P, cf, hp, o, d_out, rep);
        break;
      case PDEB200_MG_BICGSTAB:
        st = mg_bicgstab(ctx, P, cf, hp, o, d_out, rep);
        break;
      default:
        throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "unknown method"};
    }
  });
  PDEB_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
  PDEB_CUDA(cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  PDEB_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  if (rep) rep->device_ms = ms;
  return st;
}

}  // namespace pdeb
