// Reference BiCGStab and GMRES(m) on the full grid (identity boundary rows),
// MG-preconditioned BiCGStab on the folded system, and the FP32-inside-FP64
// iterative refinement of the MG forms. Scalars live in the device control
// block and are derived by the last block of each fused reduction.
#include <cmath>
#include <cstring>
#include <type_traits>

#include "host.h"
#include "solvers.cuh"

namespace pdeb {

// ------------------------------------------------------------ vector kernels

template <typename T>
__global__ void k_axpby(long long n, T* __restrict__ y, const T* __restrict__ x, double a, double b,
                        const Ctl* ctl) {  // y = a*x + b*y
  if (ctl_stopped(ctl)) return;
  for (long long t = gtid(); t < n; t += gstride()) y[t] = T(a * double(x[t]) + b * double(y[t]));
}

// r = b - A x over the full grid (identity boundary rows), sum r^2
template <class Coef, class Post>
__global__ void __launch_bounds__(kBx* kBy) k_full_resid_out(GridDev g, Coef cf, const double* __restrict__ x,
                                                             const double* __restrict__ b, double* __restrict__ r,
                                                             RedSlot slot, Post post, const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  const int chunk = (g.nz + gridDim.z - 1) / gridDim.z;
  const int k0 = blockIdx.z * chunk, k1 = min(g.nz, k0 + chunk);
  double acc[1] = {0.0};
  if (i < g.nx && j < g.ny) {
    for (int k = k0; k < k1; ++k) {
      const long long id = ((long long)k * g.ny + j) * g.nx + i;
      const bool interior = i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2 &&
                            (g.dim == 2 || (k >= 1 && k <= g.nz - 2));
      double v = x[id];
      if (interior) {
        const Stencil<double> s = cf.template at<double>(g, id);
        const double zp = g.dim == 3 ? x[id + g.sxy] : 0.0, zm = g.dim == 3 ? x[id - g.sxy] : 0.0;
        v = s.c * x[id] + nb_sum<double>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, g.dim);
      }
      const double rv = b[id] - v;
      r[id] = rv;
      acc[0] += rv * rv;
    }
  }
  grid_reduce<1, false>(acc, slot, post);
}

// ------------------------------------------------- reference BiCGStab posts

// BiCGStabSolve (src/backends/cpu/solvers/krylov.cpp:82-185)
struct PostBiRho {  // rho = rhat.r ; beta for iter > 0
  Ctl* c;
  __device__ void operator()(const double* v) const {
    const double rho = v[0];
    if (fabs(rho) < c->brk) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
      return;
    }
    c->beta = (rho / c->rho_prev) * (c->alpha / c->omega);
    c->rho = rho;
  }
};
struct PostBiAlpha {  // alpha = rho / (rhat.v)
  Ctl* c;
  __device__ void operator()(const double* v) const {
    if (fabs(v[0]) < c->brk) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
      return;
    }
    c->alpha = c->rho / v[0];
  }
};
struct PostBiS {  // |s| < tol: early exit after x += alpha p
  Ctl* c;
  int relative;
  __device__ void operator()(const double* v) const {
    const bool hit = relative ? v[0] <= c->tol2 : sqrt(v[0]) < c->tol;
    if (hit) {
      c->stop = 1;
      c->aux[1] = 1.0;
    }
  }
};
struct PostBiOmega {  // v = {t.t, t.s}
  Ctl* c;
  __device__ void operator()(const double* v) const {
    if (fabs(v[0]) < c->brk) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
      return;
    }
    c->omega = v[1] / v[0];
  }
};
struct PostBiResid {  // r = b - Ax (true residual) or s - omega t
  Ctl* c;
  int relative;
  __device__ void operator()(const double* v) const {
    c->rr = v[0];
    c->iter += 1;
    const bool hit = relative ? v[0] <= c->tol2 : sqrt(v[0]) < c->tol;
    if (hit) {
      c->done = 1;
      c->status = PDEB200_OK;
    } else if (fabs(c->omega) < c->brk) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
    } else if (c->iter >= c->max_iter) {
      c->done = 1;
      c->status = PDEB200_ERR_NOT_CONVERGED;
    } else {
      c->rho_prev = c->rho;
    }
  }
};

// p = r + beta (p - omega v)   (first: p = r)
template <typename T>
__global__ void k_bi_p(long long n, T* __restrict__ p, const T* __restrict__ r, const T* __restrict__ v, int first,
                       const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  const double beta = ctl->beta, omega = ctl->omega;
  for (long long t = gtid(); t < n; t += gstride())
    p[t] = first ? r[t] : T(double(r[t]) + beta * (double(p[t]) - omega * double(v[t])));
}

// s = r - alpha v, sum s^2
template <typename T, class Post>
__global__ void k_bi_s(long long n, T* __restrict__ s, const T* __restrict__ r, const T* __restrict__ v, RedSlot slot,
                       Post post, const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  const double alpha = ctl->alpha;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    const T sv = T(double(r[t]) - alpha * double(v[t]));
    s[t] = sv;
    acc[0] += double(sv) * double(sv);
  }
  grid_reduce<1, false>(acc, slot, post);
}

// early exit of the s-check: x += alpha p, then done
template <typename T>
__global__ void k_bi_exit(long long n, T* __restrict__ x, const T* __restrict__ p, Ctl* ctl) {
  if (ctl->done || !ctl->stop || ctl->aux[1] == 0.0) return;
  const double alpha = ctl->alpha;
  for (long long t = gtid(); t < n; t += gstride()) x[t] = T(double(x[t]) + alpha * double(p[t]));
}
__global__ void k_bi_exit_flag(Ctl* ctl) {
  if (ctl->done || !ctl->stop || ctl->aux[1] == 0.0) return;
  ctl->iter += 1;
  ctl->done = 1;
  ctl->status = PDEB200_OK;
}

// x += alpha p + omega s
template <typename T>
__global__ void k_bi_x(long long n, T* __restrict__ x, const T* __restrict__ p, const T* __restrict__ s,
                       const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  const double alpha = ctl->alpha, omega = ctl->omega;
  for (long long t = gtid(); t < n; t += gstride())
    x[t] = T(double(x[t]) + alpha * double(p[t]) + omega * double(s[t]));
}

// r = s - omega t, sum r^2 (recursive residual of the preconditioned form)
template <typename T, class Post>
__global__ void k_bi_r(long long n, T* __restrict__ r, const T* __restrict__ s, const T* __restrict__ t_,
                       RedSlot slot, Post post, const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  const double omega = ctl->omega;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    const T rv = T(double(s[t]) - omega * double(t_[t]));
    r[t] = rv;
    acc[0] += double(rv) * double(rv);
  }
  grid_reduce<1, false>(acc, slot, post);
}

// two dots in one pass: {t.t, t.s}
template <typename T, class Post>
__global__ void k_dot_tt_ts(long long n, const T* __restrict__ t_, const T* __restrict__ s, RedSlot slot, Post post,
                            const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  double acc[2] = {0.0, 0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    const double tv = double(t_[t]);
    acc[0] += tv * tv;
    acc[1] += tv * double(s[t]);
  }
  grid_reduce<2, false>(acc, slot, post);
}

struct PostBiInit {  // |r0| check and rho_prev = alpha = omega = 1
  Ctl* c;
  int relative;
  __device__ void operator()(const double* v) const {
    c->rho_prev = 1.0;
    c->alpha = 1.0;
    c->omega = 1.0;
    c->rr = v[0];
    if (relative) {
      c->bb = v[0];
      c->tol2 = c->tol * c->tol * v[0];
    }
    const bool hit = relative ? (v[0] == 0.0) : sqrt(v[0]) < c->tol;
    if (hit) {
      c->done = 1;
      c->status = PDEB200_OK;
    }
  }
};

template <typename T, class Post>
__global__ void k_dot_skip(long long n, const T* __restrict__ a, const T* __restrict__ b, RedSlot slot, Post post,
                           const Ctl* ctl) {
  if (ctl_stopped(ctl)) return;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) acc[0] += double(a[t]) * double(b[t]);
  grid_reduce<1, false>(acc, slot, post);
}

template <class Coef>
pdeb200_status bicgstab_reference(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_x,
                                  pdeb200_report* rep) {
  const GridDev& g = P.g;
  const long long n = g.n;
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  const int relative = o->tol_mode == PDEB200_TOL_RELATIVE;
  Buf buf(sizeof(double) * n * 7, ctx->stream);
  double* B = buf.as<double>();
  double *b = B, *r = B + n, *rhat = B + 2 * n, *p = B + 3 * n, *v = B + 4 * n, *s = B + 5 * n, *t = B + 6 * n;
  PDEB_CUDA(cudaMemsetAsync(B, 0, sizeof(double) * n * 7, ctx->stream));
  ctl_init(ctx, max_iter, o->tol, 1e-30);
  build_full_rhs(ctx, P, b);
  PDEB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(rhat, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  const int nb = vec_blocks(n, ctx);
  Ctl* C = ctx->d_ctl;
  k_dot<double, PostBiInit><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostBiInit{C, relative}, nullptr);
  ctx->count();
  const dim3 grid = stencil_grid_full(g), block = stencil_block();
  auto iterate = [&](int it) {
    k_dot_skip<double, PostBiRho><<<nb, 256, 0, ctx->stream>>>(n, rhat, r, ctx->slot(), PostBiRho{C}, C);
    k_bi_p<double><<<nb, 256, 0, ctx->stream>>>(n, p, r, v, it == 0, C);
    k_apply_full<Coef, 1, PostBiAlpha><<<grid, block, 0, ctx->stream>>>(g, cf, p, v, ctx->slot(), PostBiAlpha{C}, C,
                                                                         rhat);
    k_bi_s<double, PostBiS><<<nb, 256, 0, ctx->stream>>>(n, s, r, v, ctx->slot(), PostBiS{C, relative}, C);
    k_bi_exit<double><<<nb, 256, 0, ctx->stream>>>(n, d_x, p, C);
    k_bi_exit_flag<<<1, 1, 0, ctx->stream>>>(C);
    k_apply_full<Coef, 0, NoPost><<<grid, block, 0, ctx->stream>>>(g, cf, s, t, RedSlot{}, NoPost{}, C);
    k_dot_tt_ts<double, PostBiOmega><<<nb, 256, 0, ctx->stream>>>(n, t, s, ctx->slot(), PostBiOmega{C}, C);
    k_bi_x<double><<<nb, 256, 0, ctx->stream>>>(n, d_x, p, s, C);
    k_full_resid_out<Coef, PostBiResid><<<grid, block, 0, ctx->stream>>>(g, cf, d_x, b, r, ctx->slot(),
                                                                         PostBiResid{C, relative}, C);
    ctx->count(10);
  };
  pdeb200_status st = drive(ctx, o, max_iter + 1, iterate, false);
  const Ctl c = ctl_poll(ctx);
  if (rep) {
    rep->iterations = c.iter;
    rep->converged = st == PDEB200_OK;
  }
  full_residual_report(ctx, P, cf, b, d_x, r, rep);
  return st;
}

// ------------------------------------------------------- reference GMRES(m)

// GmresSolve (src/backends/cpu/solvers/krylov.cpp:187-333): modified
// Gram-Schmidt, Givens rotations, absolute tolerance on |g|. The Hessenberg
// matrix, rotations and g live in a device scalar block; the small dense work
// runs in single-thread kernels, so no host round trip per step.
struct GmresState {
  double* H;   // (m+1) x m, row-major H[i*m + j]
  double* cs;  // m
  double* sn;  // m
  double* g;   // m+1
  double* y;   // m
  int m;
  int* fail;
  int* iter_total;
  int* cycle_break;
};

struct PostStoreH {
  double* h;
  __device__ void operator()(const double* v) const { *h = v[0]; }
};

// w -= h_prev * V_prev (when prev >= 0), then sum(w * V_next) -> H[next][j]
__global__ void k_mgs_step(long long n, double* __restrict__ w, const double* __restrict__ vprev,
                           const double* __restrict__ hprev, const double* __restrict__ vnext, RedSlot slot,
                           PostStoreH post, const GmresState st) {
  if (*st.cycle_break || *st.fail) return;
  const double h = hprev ? *hprev : 0.0;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    double wv = w[t];
    if (vprev) {
      wv -= h * vprev[t];
      w[t] = wv;
    }
    if (vnext) acc[0] += wv * vnext[t];
  }
  if (vnext) grid_reduce<1, false>(acc, slot, post);
}

// H[j+1][j] = |w| (after the last MGS axpy)
__global__ void k_mgs_last(long long n, double* __restrict__ w, const double* __restrict__ vprev,
                           const double* __restrict__ hprev, RedSlot slot, PostStoreH post, const GmresState st) {
  if (*st.cycle_break || *st.fail) return;
  const double h = *hprev;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    const double wv = w[t] - h * vprev[t];
    w[t] = wv;
    acc[0] += wv * wv;
  }
  grid_reduce<1, false>(acc, slot, post);
}

// H[j+1][j] = sqrt(sum); V[j+1] = w / H[j+1][j] when positive
__global__ void k_gmres_normalize(long long n, const double* __restrict__ w, double* __restrict__ vnext,
                                  const double* __restrict__ hsq, const GmresState st) {
  if (*st.cycle_break || *st.fail) return;
  const double h = sqrt(*hsq);
  // the reference allocates V as zeros each cycle: V[j+1] stays 0 when |w| = 0
  for (long long t = gtid(); t < n; t += gstride()) vnext[t] = h > 0.0 ? w[t] / h : 0.0;
}

// Givens rotations of column j and of g; stopping test on |g[j+1]| (krylov.cpp:257-289)
__global__ void k_gmres_givens(GmresState st, int j, double tol) {
  if (*st.cycle_break || *st.fail) return;
  const int m = st.m;
  double* H = st.H;
#define HH(a, b) H[(a) * m + (b)]
  HH(j + 1, j) = sqrt(HH(j + 1, j));  // stored as a squared norm by the reduction
  for (int i = 0; i < j; ++i) {
    const double v1 = HH(i, j), v2 = HH(i + 1, j);
    HH(i, j) = st.cs[i] * v1 - st.sn[i] * v2;
    HH(i + 1, j) = st.sn[i] * v1 + st.cs[i] * v2;
  }
  const double h_j1j = HH(j + 1, j), h_jj = HH(j, j);
  const double denom = sqrt(h_jj * h_jj + h_j1j * h_j1j);
  if (denom < 1e-30) {
    *st.fail = 1;
    return;
  }
  st.cs[j] = h_jj / denom;
  st.sn[j] = -h_j1j / denom;
  HH(j, j) = st.cs[j] * h_jj - st.sn[j] * h_j1j;
  HH(j + 1, j) = 0.0;
  const double g1 = st.g[j], g2 = st.g[j + 1];
  st.g[j] = st.cs[j] * g1 - st.sn[j] * g2;
  st.g[j + 1] = st.sn[j] * g1 + st.cs[j] * g2;
  *st.iter_total += 1;
  if (fabs(st.g[j + 1]) < tol) *st.cycle_break = 1;
#undef HH
}

// back-substitution with y_dim = min(m, iter_total) (krylov.cpp:297-308)
__global__ void k_gmres_solve_y(GmresState st, int m_cycle) {
  if (*st.fail) return;
  const int m = st.m;
  const int it = *st.iter_total;
  const int y_dim = m_cycle < it ? m_cycle : it;
  for (int i = y_dim - 1; i >= 0; --i) {
    double sum = st.g[i];
    for (int k = i + 1; k < y_dim; ++k) sum -= st.H[i * m + k] * st.y[k];
    if (fabs(st.H[i * m + i]) < 1e-30) {
      *st.fail = 1;
      return;
    }
    st.y[i] = sum / st.H[i * m + i];
  }
  for (int i = y_dim; i < m; ++i) st.y[i] = 0.0;
  st.H[m * m + 0] = (double)y_dim;  // (row m, column 0) is free after the cycle: holds y_dim
}

// x += sum_j y_j V_j (j < y_dim)
__global__ void k_gmres_update_x(long long n, double* __restrict__ x, const double* __restrict__ V,
                                 const GmresState st) {
  if (*st.fail) return;
  const int y_dim = (int)st.H[st.m * st.m];
  for (long long t = gtid(); t < n; t += gstride()) {
    double v = x[t];
    for (int j = 0; j < y_dim; ++j) v += st.y[j] * V[(size_t)j * n + t];
    x[t] = v;
  }
}

__global__ void k_gmres_cycle_start(GmresState st, const double* beta_sq, double* V0scale) {
  // g = [beta, 0...], H = 0, flags reset
  const int m = st.m;
  for (int i = 0; i < (m + 1) * m; ++i) st.H[i] = 0.0;
  for (int i = 0; i <= m; ++i) st.g[i] = 0.0;
  st.g[0] = sqrt(*beta_sq);
  *st.cycle_break = 0;
  *V0scale = st.g[0];
}

__global__ void k_scale_into(long long n, double* __restrict__ dst, const double* __restrict__ src,
                             const double* __restrict__ denom) {
  const double d = *denom;
  for (long long t = gtid(); t < n; t += gstride()) dst[t] = src[t] / d;
}

struct PostStoreAt {
  double* p;
  __device__ void operator()(const double* v) const { *p = v[0]; }
};

template <class Coef>
pdeb200_status gmres_reference(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_x,
                               pdeb200_report* rep) {
  const GridDev& g = P.g;
  const long long n = g.n;
  const int restart = o->gmres_restart > 1 ? o->gmres_restart : 1;
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  const int m = restart;
  Buf vb(sizeof(double) * n * (m + 1), ctx->stream), wb(sizeof(double) * n, ctx->stream),
      bb(sizeof(double) * n, ctx->stream), rb(sizeof(double) * n, ctx->stream);
  double *V = vb.as<double>(), *w = wb.as<double>(), *b = bb.as<double>(), *r = rb.as<double>();
  // H (m+1)*m, cs m, sn m, g m+1, y m, beta^2 1, scale 1, then the int flags
  const size_t small = (size_t)(m + 1) * m + 4 * (size_t)m + 3 + 8;
  Buf sb(sizeof(double) * small + 4 * sizeof(int), ctx->stream);
  double* S = sb.as<double>();
  PDEB_CUDA(cudaMemsetAsync(S, 0, sizeof(double) * small + 4 * sizeof(int), ctx->stream));
  GmresState st;
  st.H = S;
  st.cs = S + (m + 1) * m;
  st.sn = st.cs + m;
  st.g = st.sn + m;
  st.y = st.g + m + 1;
  double* beta_sq = st.y + m;
  double* scal = beta_sq + 1;
  int* ints = reinterpret_cast<int*>(S + small);
  st.fail = ints;
  st.iter_total = ints + 1;
  st.cycle_break = ints + 2;
  st.m = m;
  const int nb = vec_blocks(n, ctx);
  const dim3 grid = stencil_grid_full(g), block = stencil_block();
  build_full_rhs(ctx, P, b);
  PDEB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, ctx->stream));
  // r = b - A*0 = b, beta^2
  PDEB_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  k_dot<double, PostStoreAt><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostStoreAt{beta_sq}, nullptr);
  ctx->count();
  double hb = 0.0;
  PDEB_CUDA(cudaMemcpyAsync(&hb, beta_sq, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
  pdeb200_status status = PDEB200_ERR_NOT_CONVERGED;
  int iter_total = 0;
  if (std::sqrt(hb) < o->tol) {
    status = PDEB200_OK;
  } else {
    while (iter_total < max_iter) {
      const int mc = std::min(restart, max_iter - iter_total);
      k_gmres_cycle_start<<<1, 1, 0, ctx->stream>>>(st, beta_sq, scal);
      k_scale_into<<<nb, 256, 0, ctx->stream>>>(n, V, r, scal);
      ctx->count(2);
      for (int j = 0; j < mc; ++j) {
        double* vj = V + (size_t)j * n;
        // w = A V_j (skips once the cycle broke)
        k_apply_full<Coef, 0, NoPost><<<grid, block, 0, ctx->stream>>>(g, cf, vj, w, RedSlot{}, NoPost{}, nullptr);
        // MGS: H[i][j] = w.V_i ; w -= H[i][j] V_i
        for (int i = 0; i <= j; ++i) {
          const double* vprev = i > 0 ? V + (size_t)(i - 1) * n : nullptr;
          const double* hprev = i > 0 ? st.H + (size_t)(i - 1) * m + j : nullptr;
          k_mgs_step<<<nb, 256, 0, ctx->stream>>>(n, w, vprev, hprev, V + (size_t)i * n, ctx->slot(),
                                                  PostStoreH{st.H + (size_t)i * m + j}, st);
        }
        k_mgs_last<<<nb, 256, 0, ctx->stream>>>(n, w, V + (size_t)j * n, st.H + (size_t)j * m + j, ctx->slot(),
                                                PostStoreH{st.H + (size_t)(j + 1) * m + j}, st);
        k_gmres_normalize<<<nb, 256, 0, ctx->stream>>>(n, w, V + (size_t)(j + 1) * n, st.H + (size_t)(j + 1) * m + j,
                                                       st);
        k_gmres_givens<<<1, 1, 0, ctx->stream>>>(st, j, o->tol);
        ctx->count(j + 5);
        if ((j & 7) == 7) {
          int flags[3];
          PDEB_CUDA(cudaMemcpyAsync(flags, ints, sizeof(flags), cudaMemcpyDeviceToHost, ctx->stream));
          PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
          if (flags[0] || flags[2]) break;
        }
      }
      k_gmres_solve_y<<<1, 1, 0, ctx->stream>>>(st, mc);
      k_gmres_update_x<<<nb, 256, 0, ctx->stream>>>(n, d_x, V, st);
      k_full_resid_out<Coef, PostStoreAt><<<grid, block, 0, ctx->stream>>>(g, cf, d_x, b, r, ctx->slot(),
                                                                           PostStoreAt{beta_sq}, nullptr);
      ctx->count(3);
      int flags[3];
      PDEB_CUDA(cudaMemcpyAsync(flags, ints, sizeof(flags), cudaMemcpyDeviceToHost, ctx->stream));
      PDEB_CUDA(cudaMemcpyAsync(&hb, beta_sq, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
      iter_total = flags[1];
      if (flags[0]) {
        status = PDEB200_ERR_BREAKDOWN;
        break;
      }
      if (std::sqrt(hb) < o->tol) {
        status = PDEB200_OK;
        break;
      }
      if (iter_total >= max_iter) break;
      if (o->cancel && *o->cancel) {
        status = PDEB200_ERR_CANCELLED;
        break;
      }
    }
  }
  if (rep) {
    rep->iterations = iter_total;
    rep->converged = status == PDEB200_OK;
  }
  full_residual_report(ctx, P, cf, b, d_x, r, rep);
  return status;
}

// ----------------------------------------------------------- MG-BiCGStab

// Right-preconditioned BiCGStab on the folded system with a V-cycle M:
//   p = r + beta(p - omega v); phat = M p; v = A phat; alpha = rho/(rhat.v)
//   s = r - alpha v; shat = M s; t = A shat; omega = (t.s)/(t.t)
//   x += alpha phat + omega shat; r = s - omega t   (relative rule on |r|)
template <class Coef, class HierT, typename T>
pdeb200_status mg_bicgstab_core(Context* ctx, HierT& H, const GridDev& g, const Coef& cf, const T* b, T* x,
                                int max_iter, double tol, const pdeb200_options* o, int* iters) {
  const long long n = g.n;
  Buf buf(sizeof(T) * n * 7, ctx->stream);
  T* B = buf.template as<T>();
  T *r = B, *rhat = B + n, *p = B + 2 * n, *v = B + 3 * n, *s = B + 4 * n, *t = B + 5 * n, *ph = B + 6 * n;
  PDEB_CUDA(cudaMemsetAsync(B, 0, sizeof(T) * n * 7, ctx->stream));
  PDEB_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  PDEB_CUDA(cudaMemcpyAsync(rhat, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, ctx->stream));
  ctl_init(ctx, max_iter, tol, 1e-300);
  Ctl* C = ctx->d_ctl;
  const int nb = vec_blocks(n, ctx);
  k_dot<T, PostBiInit><<<nb, 256, 0, ctx->stream>>>(n, r, r, ctx->slot(), PostBiInit{C, 1}, nullptr);
  ctx->count();
  const dim3 grid = stencil_grid_auto(g), block = stencil_block();
  T* z = H.z();
  auto iterate = [&](int it) {
    k_dot_skip<T, PostBiRho><<<nb, 256, 0, ctx->stream>>>(n, rhat, r, ctx->slot(), PostBiRho{C}, C);
    k_bi_p<T><<<nb, 256, 0, ctx->stream>>>(n, p, r, v, it == 0, C);
    H.vcycle(ctx, p, C);
    PDEB_CUDA(cudaMemcpyAsync(ph, z, sizeof(T) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    k_apply_folded<Coef, T, 0, NoPost><<<grid, block, 0, ctx->stream>>>(g, cf, ph, v, RedSlot{}, NoPost{}, C);
    k_dot_skip<T, PostBiAlpha><<<nb, 256, 0, ctx->stream>>>(n, rhat, v, ctx->slot(), PostBiAlpha{C}, C);
    k_bi_s<T, PostBiS><<<nb, 256, 0, ctx->stream>>>(n, s, r, v, ctx->slot(), PostBiS{C, 1}, C);
    k_bi_exit<T><<<nb, 256, 0, ctx->stream>>>(n, x, ph, C);
    k_bi_exit_flag<<<1, 1, 0, ctx->stream>>>(C);
    H.vcycle(ctx, s, C);
    k_apply_folded<Coef, T, 0, NoPost><<<grid, block, 0, ctx->stream>>>(g, cf, z, t, RedSlot{}, NoPost{}, C);
    k_dot_tt_ts<T, PostBiOmega><<<nb, 256, 0, ctx->stream>>>(n, t, s, ctx->slot(), PostBiOmega{C}, C);
    k_bi_x<T><<<nb, 256, 0, ctx->stream>>>(n, x, ph, z, C);
    k_bi_r<T, PostBiResid><<<nb, 256, 0, ctx->stream>>>(n, r, s, t, ctx->slot(), PostBiResid{C, 1}, C);
    ctx->count(12);
  };
  // iterations after the first are identical: replay them as a graph
  IterGraph graph;
  int graphed = -1;
  auto step = [&](int it) {
    if (it == 0) {
      iterate(0);
      return;
    }
    if (graphed < 0) graphed = graph.capture(ctx, [&](int) { iterate(1); }) ? 1 : 0;
    if (graphed)
      graph.launch(ctx);
    else
      iterate(it);
  };
  pdeb200_status st = drive(ctx, o, max_iter + 1, step, false);
  const Ctl c = ctl_poll(ctx);
  *iters = c.iter;
  return st;
}

template <class Coef>
pdeb200_status mg_bicgstab(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_problem* hp,
                           const pdeb200_options* o, double* d_x, pdeb200_report* rep) {
  if (o->precision == PDEB200_MIXED) return mixed_refinement(ctx, P, cf, hp, o, d_x, rep);
  const long long n = P.g.n;
  Hierarchy<Coef, double> H;
  H.build(ctx, P, hp, cf, o);
  Buf bfb(sizeof(double) * n, ctx->stream), rb(sizeof(double) * n, ctx->stream);
  double *bf = bfb.as<double>(), *r = rb.as<double>();
  build_folded_rhs(ctx, P, cf, bf);
  int it = 0;
  pdeb200_status st = mg_bicgstab_core<Coef, Hierarchy<Coef, double>, double>(
      ctx, H, P.g, cf, bf, d_x, o->max_iter > 1 ? o->max_iter : 1, o->tol, o, &it);
  if (rep) {
    rep->iterations = it;
    rep->converged = st == PDEB200_OK;
  }
  folded_residual_report(ctx, P, cf, bf, d_x, r, rep);
  fill_boundary(ctx, P.g, d_x, nullptr);
  return st;
}

// ------------------------------------------------- mixed precision (IR)

// The inner operator in FP32: constant stencils convert, sampled k is stored
// in FP32 (or BF16 for the smoother hierarchy when requested).
template <class Coef>
struct Lower;
template <>
struct Lower<CoefConst> {
  using F32 = CoefConst;
  using S16 = CoefConst;
  static F32 make32(Context*, DevProblem&, const CoefConst& c, std::vector<Buf>*) { return c; }
  static S16 make16(Context*, DevProblem&, const CoefConst& c, std::vector<Buf>*) { return c; }
};
template <>
struct Lower<CoefDivk<double>> {
  using F32 = CoefDivk<float>;
  using S16 = CoefDivk<__nv_bfloat16>;
  template <typename KT>
  static CoefDivk<KT> conv(Context* ctx, DevProblem& P, const CoefDivk<double>& c, std::vector<Buf>* owned) {
    owned->emplace_back(sizeof(KT) * P.g.n, ctx->stream);
    KT* k = owned->back().template as<KT>();
    k_convert<KT, double><<<vec_blocks(P.g.n, ctx), 256, 0, ctx->stream>>>(P.g.n, k, c.k);
    ctx->count();
    CoefDivk<KT> o;
    o.k = k;
    o.ihx2 = c.ihx2;
    o.ihy2 = c.ihy2;
    o.ihz2 = c.ihz2;
    o.cx = c.cx;
    o.dyc = c.dyc;
    o.dzc = c.dzc;
    o.e = c.e;
    return o;
  }
  static F32 make32(Context* ctx, DevProblem& P, const CoefDivk<double>& c, std::vector<Buf>* owned) {
    return conv<float>(ctx, P, c, owned);
  }
  static S16 make16(Context* ctx, DevProblem& P, const CoefDivk<double>& c, std::vector<Buf>* owned) {
    return conv<__nv_bfloat16>(ctx, P, c, owned);
  }
};

// r = b - A x in FP64 (folded), |r|^2 ; optional scaled FP32 copy r32 = r / |r|
struct PostRRtoAux {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->rr = v[0];
    c->aux[2] = sqrt(v[0]);
  }
};

template <typename T>
__global__ void k_scale_to(long long n, T* __restrict__ dst, const double* __restrict__ src, const Ctl* ctl) {
  const double s = ctl->aux[2] > 0 ? 1.0 / ctl->aux[2] : 0.0;
  for (long long t = gtid(); t < n; t += gstride()) dst[t] = T(src[t] * s);
}

template <typename T>
__global__ void k_add_scaled(long long n, double* __restrict__ x, const T* __restrict__ e, const Ctl* ctl) {
  const double s = ctl->aux[2];
  for (long long t = gtid(); t < n; t += gstride()) x[t] += s * double(e[t]);
}

// MG-PCG core in precision T (relative rule on the recursive residual). One
// object serves every outer step of a refinement: its vectors and the
// captured iteration (the same b, x and hierarchy buffers each time) are made
// once, so later steps neither allocate nor capture.
template <class Coef, class HierT, typename T>
struct MgPcgCore {
  Buf buf;
  IterGraph graph;
  int graphed = -1;  // -1: not captured yet
  bool fused_dot = false;

  pdeb200_status run(Context* ctx, HierT& H, const GridDev& g, const Coef& cf, const T* b, T* x, int max_iter,
                     double tol, const pdeb200_options* o, int* iters) {
    const long long n = g.n;
    if (!buf.bytes()) buf = Buf(sizeof(T) * n * 3, ctx->stream);
    T* B = buf.template as<T>();
    T *r = B, *p = B + n, *q = B + 2 * n;
    PDEB_CUDA(cudaMemsetAsync(B, 0, sizeof(T) * n * 3, ctx->stream));
    PDEB_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, ctx->stream));
    PDEB_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    ctl_init(ctx, max_iter, tol, 1e-300);
    Ctl* C = ctx->d_ctl;
    const int nb = vec_blocks(n, ctx);
    k_dot<T, PostBB><<<nb, 256, 0, ctx->stream>>>(n, b, b, ctx->slot(), PostBB{C}, C);
    T* z = H.z();
    H.vcycle(ctx, r, C);
    k_dot<T, PostRZ><<<nb, 256, 0, ctx->stream>>>(n, r, z, ctx->slot(), PostRZ{C}, C);
    k_cg_p<T><<<nb, 256, 0, ctx->stream>>>(n, p, z, C, 1);
    ctx->count(3);
    const dim3 grid = stencil_grid_auto(g), block = stencil_block();
    auto iterate = [&](int) {
      k_apply_folded<Coef, T, 1, PostAlpha><<<grid, block, 0, ctx->stream>>>(g, cf, p, q, ctx->slot(), PostAlpha{C}, C);
      k_cg_xr<T, PostRRRel><<<nb, 256, 0, ctx->stream>>>(n, x, r, p, q, ctx->slot(), PostRRRel{C}, C);
      // beta from r.z summed by the preconditioner's last colour passes when it can
      if (!H.vcycle_dot(ctx, r, C, ctx->slot())) {
        k_dot<T, PostBeta><<<nb, 256, 0, ctx->stream>>>(n, r, z, ctx->slot(), PostBeta{C}, C);
        ctx->count();
      }
      k_cg_p<T><<<nb, 256, 0, ctx->stream>>>(n, p, z, C, 0);
      ctx->count(3);
    };
    if (graphed < 0) graphed = graph.capture(ctx, iterate) ? 1 : 0;
    auto step = [&](int it) {
      if (graphed)
        graph.launch(ctx);
      else
        iterate(it);
    };
    pdeb200_status st = drive(ctx, o, max_iter + 1, step, false);
    const Ctl c = ctl_poll(ctx);
    *iters = c.iter;
    return st;
  }
};

// FP64 iterative refinement around an FP32 MG-preconditioned Krylov solve:
// r = b - A x in FP64; e = solve(A e = r/|r|) in FP32 to inner_tol; x += |r| e.
// FP64 is kept for the outer residual, the update and the report.
template <class Coef>
pdeb200_status mixed_refinement(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_problem* hp,
                                const pdeb200_options* o, double* d_x, pdeb200_report* rep) {
  if constexpr (std::is_same<Coef, CoefNodal>::value) {
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "mixed precision supports constant and divergence-form k"};
  } else {
    using L = Lower<Coef>;
    const GridDev& g = P.g;
    const long long n = g.n;
    std::vector<Buf> owned;
    typename L::F32 cf32 = L::make32(ctx, P, cf, &owned);
    Buf bfb(sizeof(double) * n, ctx->stream), rb(sizeof(double) * n, ctx->stream), r32b(sizeof(float) * n, ctx->stream),
        e32b(sizeof(float) * n, ctx->stream);
    double *bf = bfb.as<double>(), *r = rb.as<double>();
    float *r32 = r32b.as<float>(), *e32 = e32b.as<float>();
    PDEB_CUDA(cudaMemsetAsync(r, 0, sizeof(double) * n, ctx->stream));
    build_folded_rhs(ctx, P, cf, bf);
    PDEB_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, ctx->stream));
    const bool nonsym = o->method == PDEB200_MG_BICGSTAB;
    pdeb200_options io = *o;
    io.tol = o->inner_tol > 0 ? o->inner_tol : 1e-5;
    io.precision = PDEB200_FP64;
    const int max_outer = o->max_outer > 0 ? o->max_outer : 50;
    const int nb = vec_blocks(n, ctx);
    const dim3 grid = stencil_grid_auto(g), block = stencil_block();
    Ctl* C = ctx->d_ctl;
    // |b|^2
    k_dot<double, PostBBOnly><<<nb, 256, 0, ctx->stream>>>(n, bf, bf, ctx->slot(), PostBBOnly{C}, nullptr);
    ctx->count();
    const double bnorm = std::sqrt(ctl_poll(ctx).bb);
    int total_inner = 0, outer = 0;
    pdeb200_status st = PDEB200_ERR_NOT_CONVERGED;
    double rel = 1.0;
    auto run = [&](auto& H) {
      using HT = std::decay_t<decltype(H)>;
      MgPcgCore<typename L::F32, HT, float> pcg;
      for (outer = 0; outer < max_outer; ++outer) {
        k_residual_folded<Coef, double, double, 1, PostRRtoAux><<<grid, block, 0, ctx->stream>>>(
            g, cf, d_x, bf, r, ctx->slot(), PostRRtoAux{C}, nullptr);
        ctx->count();
        const Ctl c = ctl_poll(ctx);
        rel = bnorm > 0 ? std::sqrt(c.rr) / bnorm : 0.0;
        if (rel <= o->tol || bnorm == 0.0) {
          st = PDEB200_OK;
          break;
        }
        if (o->cancel && *o->cancel) {
          st = PDEB200_ERR_CANCELLED;
          break;
        }
        k_scale_to<float><<<nb, 256, 0, ctx->stream>>>(n, r32, r, C);
        ctx->count();
        int it = 0;
        pdeb200_status is;
        // the inner solve overwrites the control block: keep |r| for the update
        const double rn = c.aux[2];
        // the inner solve only has to take the residual from `rel` to the
        // target; on the last outer step that is less than inner_tol (a factor
        // 4 of margin covers the FP32 operator's rounding)
        const double step_tol = std::max(io.tol, std::min(0.1, 0.25 * o->tol / rel));
        if (nonsym)
          is = mg_bicgstab_core<typename L::F32, HT, float>(ctx, H, g, cf32, r32, e32, io.max_iter, step_tol, &io,
                                                            &it);
        else
          is = pcg.run(ctx, H, g, cf32, r32, e32, io.max_iter, step_tol, &io, &it);
        total_inner += it;
        if (is == PDEB200_ERR_BREAKDOWN && it == 0) {
          st = PDEB200_ERR_BREAKDOWN;
          break;
        }
        std::memset(ctx->h_ctl, 0, sizeof(Ctl));
        ctx->h_ctl->aux[2] = rn;
        PDEB_CUDA(cudaMemcpyAsync(C, ctx->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, ctx->stream));
        k_add_scaled<float><<<nb, 256, 0, ctx->stream>>>(n, d_x, e32, C);
        ctx->count();
        PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
      }
    };
    if (o->bf16_coefficients && !std::is_same<Coef, CoefConst>::value) {
      // BF16 k in the smoother hierarchy; the Krylov operator stays FP32
      typename L::S16 cf16 = L::make16(ctx, P, cf, &owned);
      Hierarchy<typename L::S16, float> H16;
      H16.build(ctx, P, hp, cf16, &io);
      run(H16);
    } else {
      Hierarchy<typename L::F32, float> H;
      H.build(ctx, P, hp, cf32, &io);
      run(H);
    }
    if (rep) {
      rep->iterations = total_inner;
      rep->outer_iterations = outer;
      rep->converged = st == PDEB200_OK;
    }
    folded_residual_report(ctx, P, cf, bf, d_x, r, rep);
    fill_boundary(ctx, g, d_x, nullptr);
    return st;
  }
}

#define INST(C)                                                                                                 \
  template pdeb200_status bicgstab_reference<C>(Context*, DevProblem&, const C&, const pdeb200_options*, double*, \
                                                pdeb200_report*);                                               \
  template pdeb200_status gmres_reference<C>(Context*, DevProblem&, const C&, const pdeb200_options*, double*,  \
                                             pdeb200_report*);                                                  \
  template pdeb200_status mixed_refinement<C>(Context*, DevProblem&, const C&, const pdeb200_problem*,          \
                                              const pdeb200_options*, double*, pdeb200_report*);                \
  template pdeb200_status mg_bicgstab<C>(Context*, DevProblem&, const C&, const pdeb200_problem*,               \
                                         const pdeb200_options*, double*, pdeb200_report*);
INST(CoefConst)
INST(CoefDivk<double>)
INST(CoefNodal)

}  // namespace pdeb
