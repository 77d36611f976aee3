// Lexicographic Gauss-Seidel / SOR and the reference's single V-cycle "mg",
// reproduced exactly on the GPU.
//
// The reference sweeps in place in lexicographic order (k, j, i)
// (src/backends/cpu/solvers/relaxation.cpp:167-289, solver.cpp:808-962): a node
// reads its lower neighbours already updated and its upper neighbours not yet.
// All nodes of one hyperplane i+j+k = d depend only on hyperplanes d-1 and d+1,
// so visiting hyperplanes in increasing d (nodes of a hyperplane in parallel)
// performs exactly the reference's updates in a different but equivalent order.
//
// Small grids run the whole solve in one resident block: boundary closures,
// the sweeps, the max|du| reduction and the stopping test stay on chip and no
// block waits on another. Large grids launch one kernel per hyperplane.
#include <cmath>
#include <cstring>

#include "host.h"
#include "solvers.cuh"

namespace pdeb {

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// In-block boundary fill (same closure chain as k_fill_boundary).
__device__ void block_fill_boundary(const GridDev& g, double* u, bool dirichlet_last) {
  const long long nxy = (long long)g.nx * g.ny, nyz = (long long)g.ny * g.nz, nxz = (long long)g.nx * g.nz;
  const long long total = 2 * nyz + 2 * nxz + (g.dim == 3 ? 2 * nxy : 0);
  for (long long t = threadIdx.x; t < total; t += blockDim.x) {
    int i, j, k, f;
    long long r = t;
    if (r < 2 * nyz) {
      f = r < nyz ? kLeft : kRight;
      r %= nyz;
      j = int(r % g.ny);
      k = int(r / g.ny);
      i = f == kLeft ? 0 : g.nx - 1;
    } else if ((r -= 2 * nyz) < 2 * nxz) {
      f = r < nxz ? kBottom : kTop;
      r %= nxz;
      i = int(r % g.nx);
      k = int(r / g.nx);
      j = f == kBottom ? 0 : g.ny - 1;
    } else {
      r -= 2 * nxz;
      f = r < nxy ? kFront : kBack;
      r %= nxy;
      i = int(r % g.nx);
      j = int(r / g.nx);
      k = f == kFront ? 0 : g.nz - 1;
    }
    const bool on[6] = {i == 0, i == g.nx - 1, j == 0, j == g.ny - 1, g.dim == 3 && k == 0,
                        g.dim == 3 && k == g.nz - 1};
    int owner = -1;
    for (int q = 0; q < 6; ++q)
      if (on[q]) {
        owner = q;
        break;
      }
    if (owner != f) continue;
    u[((long long)k * g.ny + j) * g.nx + i] = boundary_final(g, u, i, j, k, dirichlet_last);
  }
}

// One node of the reference sweep: rhs = -(f + nonlinear(old)) - (lap);
// upd = rhs/center; SOR: (1-omega)*old + omega*upd (relaxation.cpp:217-276,
// solver.cpp:884-962).
template <class Coef>
__device__ __forceinline__ double lex_update(const GridDev& g, const Coef& cf, const double* __restrict__ f,
                                             double fc, const NonlinDev& nl, double* u, int i, int j, int k,
                                             double omega, double* delta, int* degenerate) {
  const long long id = ((long long)k * g.ny + j) * g.nx + i;
  const Stencil<double> s = cf.template at<double>(g, id);
  if (fabs(s.c) < 1e-12) {
    *degenerate = 1;
    return 0.0;
  }
  const double old_u = u[id];
  const double zp = g.dim == 3 ? u[id + g.sxy] : 0.0, zm = g.dim == 3 ? u[id - g.sxy] : 0.0;
  const double lap = nb_sum<double>(s, u[id + 1], u[id - 1], u[id + g.nx], u[id - g.nx], zp, zm, g.dim);
  const double rhs = -f_plus_nl(f ? f[id] : fc, nl, old_u) - lap;
  const double upd = __ddiv_rn(rhs, s.c);
  const double updated = (1.0 - omega) * old_u + omega * upd;
  u[id] = updated;
  *delta = fmax(*delta, fabs(updated - old_u));
  return updated;
}

// Visit the interior nodes of hyperplane d with stride `step` from `start`.
template <class Fn>
__device__ __forceinline__ void for_hyperplane(const GridDev& g, int d, long long start, long long step, Fn&& fn) {
  if (g.dim == 2) {
    const int jlo = max(1, d - (g.nx - 2)), jhi = min(g.ny - 2, d - 1);
    for (long long t = start; t <= jhi - jlo; t += step) {
      const int j = jlo + int(t);
      fn(d - j, j, 0);
    }
  } else {
    // (j, k) pairs with i = d - j - k in [1, nx-2]
    const int klo = max(1, d - (g.nx - 2) - (g.ny - 2)), khi = min(g.nz - 2, d - 2);
    if (khi < klo) return;
    const long long nk = khi - klo + 1;
    const long long nj = g.ny - 2;
    for (long long t = start; t < nk * nj; t += step) {
      const int k = klo + int(t / nj), j = 1 + int(t % nj);
      const int i = d - j - k;
      if (i >= 1 && i <= g.nx - 2) fn(i, j, k);
    }
  }
}

__device__ __forceinline__ int hyper_lo(const GridDev& g) { return g.dim == 3 ? 3 : 2; }
__device__ __forceinline__ int hyper_hi(const GridDev& g) {
  return g.dim == 3 ? (g.nx - 2) + (g.ny - 2) + (g.nz - 2) : (g.nx - 2) + (g.ny - 2);
}

// Whole GS/SOR solve in one block. Iteration sequence of the reference:
// 2D closures then sweep (relaxation.cpp:134-289); 3D sweep then closures
// (solver.cpp:769-981; the initial closures are applied by the host).
template <class Coef>
__global__ void __launch_bounds__(1024) k_gs_lex_block(GridDev g, Coef cf, const double* __restrict__ f, double fc,
                                                       NonlinDev nl, double* u, double omega, double tol, int max_iter,
                                                       unsigned long long budget_ns, Ctl* ctl) {
  __shared__ double red[32];
  __shared__ int s_stop;
  __shared__ int s_degen;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_stop = 0;
    s_degen = 0;
  }
  __syncthreads();
  const unsigned long long t0 = globaltimer_ns();
  int it = 0, status = PDEB200_ERR_NOT_CONVERGED;
  double delta_out = 0.0;
  for (it = 0; it < max_iter; ++it) {
    if (g.dim == 2) {
      block_fill_boundary(g, u, false);  // Neumann/Robin closures only (relaxation.cpp:135)
      __syncthreads();
    }
    double delta = 0.0;
    int degen = 0;
    const int dlo = hyper_lo(g), dhi = hyper_hi(g);
    for (int d = dlo; d <= dhi; ++d) {
      for_hyperplane(g, d, tid, blockDim.x,
                     [&](int i, int j, int k) { lex_update(g, cf, f, fc, nl, u, i, j, k, omega, &delta, &degen); });
      __syncthreads();
    }
    if (degen) s_degen = 1;
    // block max of delta
    for (int off = 16; off > 0; off >>= 1) delta = fmax(delta, __shfl_down_sync(0xffffffffu, delta, off));
    if ((tid & 31) == 0) red[tid >> 5] = delta;
    __syncthreads();
    if (tid < 32) {
      double v = tid < (int)(blockDim.x + 31) / 32 ? red[tid] : 0.0;
      for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
      if (tid == 0) red[0] = v;
    }
    __syncthreads();
    const double md = red[0];
    if (g.dim == 3) {
      block_fill_boundary(g, u, true);
      __syncthreads();
    }
    delta_out = md;
    if (tid == 0) {
      if (s_degen) s_stop = 2;
      else if (md < tol) s_stop = 1;
      else if (globaltimer_ns() - t0 > budget_ns) s_stop = 3;
    }
    __syncthreads();
    if (s_stop) break;
  }
  if (tid == 0) {
    const int stop = s_stop;
    if (stop == 1) status = PDEB200_OK;
    else if (stop == 2) status = PDEB200_ERR_DEGENERATE;
    else if (stop == 3) status = PDEB200_ERR_TIMEOUT;
    ctl->iter = stop ? it + 1 : it;
    ctl->delta = delta_out;
    ctl->status = status;
    ctl->done = 1;
  }
}

// Multi-block form: one launch per hyperplane; max|du| through an atomic max
// on the (non-negative) double's bit pattern in ctl->aux[0].
template <class Coef>
__global__ void k_gs_lex_plane(GridDev g, Coef cf, const double* __restrict__ f, double fc, NonlinDev nl, double* u,
                               double omega, int d, Ctl* ctl, int* degenerate) {
  if (ctl_stopped(ctl)) return;
  double delta = 0.0;
  int degen = 0;
  for_hyperplane(g, d, gtid(), gstride(),
                 [&](int i, int j, int k) { lex_update(g, cf, f, fc, nl, u, i, j, k, omega, &delta, &degen); });
  if (degen) *degenerate = 1;
  for (int off = 16; off > 0; off >>= 1) delta = fmax(delta, __shfl_down_sync(0xffffffffu, delta, off));
  if ((threadIdx.x & 31) == 0 && delta > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(&ctl->aux[0]), (unsigned long long)__double_as_longlong(delta));
}

// end of a multi-block sweep: stopping test of the reference
__global__ void k_gs_lex_check(Ctl* ctl, double tol) {
  if (ctl_stopped(ctl)) return;
  const double md = ctl->aux[0];
  ctl->delta = md;
  ctl->iter += 1;
  ctl->aux[0] = 0.0;
  if (md < tol) {
    ctl->stop = 1;
    ctl->status = PDEB200_OK;
  } else if (ctl->iter >= ctl->max_iter) {
    ctl->stop = 1;
    ctl->status = PDEB200_ERR_NOT_CONVERGED;
  }
}

template <class Coef>
pdeb200_status gauss_seidel(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_out,
                            pdeb200_report* rep) {
  const GridDev& g = P.g;
  const double omega = o->method == PDEB200_SOR ? o->sor_omega : 1.0;
  if (o->method == PDEB200_SOR && (omega <= 0.0 || omega >= 2.0))
    throw StatusFailure{PDEB200_ERR_INVALID, "SOR omega must be in (0,2)"};
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  PDEB_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * g.n, ctx->stream));
  ctl_init(ctx, max_iter, o->tol, 0.0);
  fill_boundary(ctx, g, d_out, nullptr);  // initial closures
  const long long interior = (long long)(g.nx - 2) * (g.ny - 2) * (g.dim == 3 ? g.nz - 2 : 1);
  if (o->gs_ordering == PDEB200_ORDER_REDBLACK)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "red-black ordering is offered through the MG forms"};
  if (interior <= (1LL << 18)) {
    const unsigned long long budget = 60ULL * 1000000000ULL;  // device-time guard: 60 s
    k_gs_lex_block<Coef><<<1, 1024, 0, ctx->stream>>>(g, cf, P.f, P.f_const, P.nl, d_out, omega, o->tol, max_iter,
                                                      budget,
                                                      ctx->d_ctl);
    ctx->count();
    const Ctl& c = ctl_poll(ctx);
    if (rep) {
      rep->iterations = c.iter;
      rep->last_delta = c.delta;
      rep->converged = c.status == PDEB200_OK;
    }
    return (pdeb200_status)c.status;
  }
  Buf degen(sizeof(int), ctx->stream);
  PDEB_CUDA(cudaMemsetAsync(degen.as<int>(), 0, sizeof(int), ctx->stream));
  int dlo = g.dim == 3 ? 3 : 2;
  int dhi = g.dim == 3 ? (g.nx - 2) + (g.ny - 2) + (g.nz - 2) : (g.nx - 2) + (g.ny - 2);
  auto iterate = [&](int) {
    if (g.dim == 2) fill_boundary(ctx, g, d_out, ctx->d_ctl, false);
    for (int d = dlo; d <= dhi; ++d) {
      k_gs_lex_plane<Coef><<<vec_blocks((long long)(g.ny) * g.nz, ctx), 256, 0, ctx->stream>>>(
          g, cf, P.f, P.f_const, P.nl, d_out, omega, d, ctx->d_ctl, degen.as<int>());
    }
    ctx->count(dhi - dlo + 1);
    if (g.dim == 3) fill_boundary(ctx, g, d_out, ctx->d_ctl);
    k_gs_lex_check<<<1, 1, 0, ctx->stream>>>(ctx->d_ctl, o->tol);
    ctx->count();
  };
  pdeb200_status st = drive(ctx, o, max_iter, iterate, true);
  const Ctl c = ctl_poll(ctx);
  int dg = 0;
  PDEB_CUDA(cudaMemcpy(&dg, degen.as<int>(), sizeof(int), cudaMemcpyDeviceToHost));
  if (dg) return PDEB200_ERR_DEGENERATE;
  if (rep) {
    rep->iterations = c.iter;
    rep->last_delta = c.delta;
    rep->converged = st == PDEB200_OK;
  }
  return st;
}

template pdeb200_status gauss_seidel<CoefConst>(Context*, DevProblem&, const CoefConst&, const pdeb200_options*,
                                                double*, pdeb200_report*);
template pdeb200_status gauss_seidel<CoefDivk<double>>(Context*, DevProblem&, const CoefDivk<double>&,
                                                       const pdeb200_options*, double*, pdeb200_report*);
template pdeb200_status gauss_seidel<CoefNodal>(Context*, DevProblem&, const CoefNodal&, const pdeb200_options*,
                                                double*, pdeb200_report*);

// ------------------------------------------------ reference single V-cycle

// MultigridVcyclePoisson (src/backends/cpu/solvers/multigrid.cpp:121-222):
// 2D, constant a, b, e, lexicographic GS smoother, full weighting on interior
// coarse nodes, bilinear prolongation-add over the whole fine grid, exactly
// one cycle. Each grid is a Level2 on the device.
struct MgRefLevel {
  int nx, ny;
  double ax, by, center;
  double *u, *b, *r;
};

// SmoothGsPoisson (multigrid.cpp:69-94), hyperplane order, one block
__global__ void __launch_bounds__(1024) k_mgref_smooth(MgRefLevel L, int iters) {
  const int tid = threadIdx.x;
  const int nx = L.nx, ny = L.ny;
  for (int it = 0; it < iters; ++it) {
    for (int d = 2; d <= (nx - 2) + (ny - 2); ++d) {
      const int jlo = max(1, d - (nx - 2)), jhi = min(ny - 2, d - 1);
      for (int t = tid; t <= jhi - jlo; t += blockDim.x) {
        const int j = jlo + t, i = d - j;
        const long long id = (long long)j * nx + i;
        const double rhs = L.b[id] - L.ax * (L.u[id - 1] + L.u[id + 1]) - L.by * (L.u[id - nx] + L.u[id + nx]);
        L.u[id] = __ddiv_rn(rhs, L.center);
      }
      __syncthreads();
    }
  }
}

// ResidualPoisson (multigrid.cpp:96-119): r = b - (center*u + ax*(ul+ur) + by*(ud+uu)) inside, 0 on the boundary
__global__ void k_mgref_residual(MgRefLevel L) {
  const long long n = (long long)L.nx * L.ny;
  for (long long t = gtid(); t < n; t += gstride()) {
    const int i = int(t % L.nx), j = int(t / L.nx);
    if (i == 0 || j == 0 || i == L.nx - 1 || j == L.ny - 1) {
      L.r[t] = 0.0;
      continue;
    }
    const double Au = L.center * L.u[t] + L.ax * (L.u[t - 1] + L.u[t + 1]) + L.by * (L.u[t - L.nx] + L.u[t + L.nx]);
    L.r[t] = L.b[t] - Au;
  }
}

// RestrictFullWeighting (multigrid.cpp:14-36): interior coarse nodes, boundary 0
__global__ void k_mgref_restrict(MgRefLevel F, MgRefLevel C) {
  const long long n = (long long)C.nx * C.ny;
  for (long long t = gtid(); t < n; t += gstride()) {
    const int ic = int(t % C.nx), jc = int(t / C.nx);
    if (ic == 0 || jc == 0 || ic == C.nx - 1 || jc == C.ny - 1) {
      C.b[t] = 0.0;
      C.u[t] = 0.0;
      continue;
    }
    const int ifx = 2 * ic, jf = 2 * jc, fx = F.nx;
    const double* fr = F.r;
    const double c = fr[(long long)jf * fx + ifx] * 0.25;
    const double e = (fr[(long long)jf * fx + ifx - 1] + fr[(long long)jf * fx + ifx + 1] +
                      fr[(long long)(jf - 1) * fx + ifx] + fr[(long long)(jf + 1) * fx + ifx]) * 0.125;
    const double dd = (fr[(long long)(jf - 1) * fx + ifx - 1] + fr[(long long)(jf - 1) * fx + ifx + 1] +
                       fr[(long long)(jf + 1) * fx + ifx - 1] + fr[(long long)(jf + 1) * fx + ifx + 1]) * 0.0625;
    C.b[t] = c + e + dd;
    C.u[t] = 0.0;
  }
}

// ProlongBilinearAdd (multigrid.cpp:38-67) as a gather: fine node (2ic+a,
// 2jc+b) receives exactly one term, from coarse node (ic,jc).
__global__ void k_mgref_prolong(MgRefLevel C, MgRefLevel F) {
  const long long n = (long long)F.nx * F.ny;
  for (long long t = gtid(); t < n; t += gstride()) {
    const int i = int(t % F.nx), j = int(t / F.nx);
    const int ic = i >> 1, jc = j >> 1;
    if (ic >= C.nx || jc >= C.ny) continue;
    const double* cu = C.u;
    const double vc = cu[(long long)jc * C.nx + ic];
    const bool ox = i & 1, oy = j & 1;
    double add;
    if (!ox && !oy) {
      add = vc;
    } else if (ox && !oy) {
      if (!(ic + 1 < C.nx)) continue;
      add = 0.5 * (vc + cu[(long long)jc * C.nx + ic + 1]);
    } else if (!ox && oy) {
      if (!(jc + 1 < C.ny)) continue;
      add = 0.5 * (vc + cu[(long long)(jc + 1) * C.nx + ic]);
    } else {
      if (!(ic + 1 < C.nx && jc + 1 < C.ny)) continue;
      const double vru = cu[(long long)(jc + 1) * C.nx + ic + 1];
      const double vr = cu[(long long)jc * C.nx + ic + 1];
      const double vu = cu[(long long)(jc + 1) * C.nx + ic];
      add = 0.25 * (vc + vr + vu + vru);
    }
    F.u[t] += add;
  }
}

pdeb200_status mg_vcycle_reference(Context* ctx, DevProblem& P, const pdeb200_problem* hp, const pdeb200_options* o,
                                   double* d_out, pdeb200_report* rep) {
  const GridDev& g = P.g;
  if (g.dim != 2 || P.coef_kind != kConst || std::fabs(P.c) > 1e-12 || std::fabs(P.d) > 1e-12)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "Multigrid requires no convection, mixed, or higher-order derivatives"};
  for (int f = 0; f < 4; ++f)
    if (g.face[f].kind != kDirichlet)
      throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "Multigrid requires Dirichlet boundaries on all sides"};
  auto can = [](int nx, int ny) { return nx >= 5 && (nx & 1) && ny >= 5 && (ny & 1); };
  if (!can(g.nx, g.ny)) throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "CPU multigrid solver failed"};
  std::vector<MgRefLevel> lv;
  std::vector<Buf> owned;
  auto coeffs = [&](MgRefLevel& L) {
    const double dx = (hp->xmax - hp->xmin) / (double)(L.nx - 1);
    const double dy = (hp->ymax - hp->ymin) / (double)(L.ny - 1);
    L.ax = hp->a / (dx * dx);
    L.by = hp->b / (dy * dy);
    L.center = -2.0 * L.ax - 2.0 * L.by + hp->e;
  };
  MgRefLevel L0{g.nx, g.ny, 0, 0, 0, d_out, nullptr, nullptr};
  owned.emplace_back(sizeof(double) * g.n, ctx->stream);
  L0.b = owned.back().as<double>();
  owned.emplace_back(sizeof(double) * g.n, ctx->stream);
  L0.r = owned.back().as<double>();
  coeffs(L0);
  lv.push_back(L0);
  const int max_levels = o->mg_max_levels;
  while ((int)lv.size() < max_levels) {
    const MgRefLevel& pr = lv.back();
    if (!can(pr.nx, pr.ny)) break;
    const int ncx = (pr.nx + 1) / 2, ncy = (pr.ny + 1) / 2;
    if (ncx < 3 || ncy < 3) break;
    MgRefLevel c{ncx, ncy, 0, 0, 0, nullptr, nullptr, nullptr};
    for (double** p : {&c.u, &c.b, &c.r}) {
      owned.emplace_back(sizeof(double) * ncx * ncy, ctx->stream);
      *p = owned.back().as<double>();
      PDEB_CUDA(cudaMemsetAsync(*p, 0, sizeof(double) * ncx * ncy, ctx->stream));
    }
    coeffs(c);
    lv.push_back(c);
    if (ncx <= 5 || ncy <= 5) break;
  }
  for (auto& L : lv)
    if (std::fabs(L.center) < 1e-12) throw StatusFailure{PDEB200_ERR_DEGENERATE, "CPU multigrid solver failed"};
  // b = BuildRhs2D, u = Dirichlet closure of zero
  build_full_rhs(ctx, P, L0.b);
  PDEB_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * g.n, ctx->stream));
  fill_boundary(ctx, g, d_out, nullptr);
  const int L = (int)lv.size();
  const int pre = o->mg_pre_smooth > 0 ? o->mg_pre_smooth : 0;
  const int post = o->mg_post_smooth > 0 ? o->mg_post_smooth : 0;
  const int coarse = o->mg_coarse_iters > 1 ? o->mg_coarse_iters : 1;
  for (int l = 0; l < L - 1; ++l) {
    k_mgref_smooth<<<1, 1024, 0, ctx->stream>>>(lv[l], pre);
    k_mgref_residual<<<vec_blocks((long long)lv[l].nx * lv[l].ny, ctx), 256, 0, ctx->stream>>>(lv[l]);
    k_mgref_restrict<<<vec_blocks((long long)lv[l + 1].nx * lv[l + 1].ny, ctx), 256, 0, ctx->stream>>>(lv[l],
                                                                                                      lv[l + 1]);
    ctx->count(3);
  }
  k_mgref_smooth<<<1, 1024, 0, ctx->stream>>>(lv[L - 1], coarse);
  ctx->count();
  for (int l = L - 2; l >= 0; --l) {
    k_mgref_prolong<<<vec_blocks((long long)lv[l].nx * lv[l].ny, ctx), 256, 0, ctx->stream>>>(lv[l + 1], lv[l]);
    k_mgref_smooth<<<1, 1024, 0, ctx->stream>>>(lv[l], post);
    ctx->count(2);
  }
  if (rep) {
    rep->iterations = 1;
    rep->converged = 1;
  }
  return PDEB200_OK;
}

}  // namespace pdeb
