// Templates shared by the solver drivers: device-side post functors of the
// fused reductions, the enqueue/poll driver, the geometric MG hierarchy with
// its V-cycle, right-hand-side builders and residual reports.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "host.h"
#include "march.cuh"
#include "sweep.cuh"

namespace pdeb {

// ------------------------------------------------------------------ posts

struct PostBBOnly {
  Ctl* c;
  __device__ void operator()(const double* v) const { c->bb = v[0]; }
};

struct PostStoreRR {
  Ctl* c;
  __device__ void operator()(const double* v) const { c->rr = v[0]; }
};

// alpha = rz / pq  (breakdown when |pq| < brk or not finite)
struct PostAlpha {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->pq = v[0];
    if (!(fabs(v[0]) >= c->brk) || isnan(v[0])) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
      return;
    }
    c->alpha = c->rz / v[0];
  }
};

// relative rule on |r|^2 <= tol2
struct PostRRRel {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->rr = v[0];
    c->iter += 1;
    if (v[0] <= c->tol2) {
      c->done = 1;
      c->status = PDEB200_OK;
    } else if (isnan(v[0])) {
      c->done = 1;
      c->status = PDEB200_ERR_BREAKDOWN;
    } else if (c->iter >= c->max_iter) {
      c->done = 1;
      c->status = PDEB200_ERR_NOT_CONVERGED;
    }
  }
};

// reference CG (krylov.cpp:58-77): stop when sqrt(rr_new) < tol, else
// beta = rr_new/rr and rr = rr_new
struct PostRRRefCG {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->rr = v[0];
    c->iter += 1;
    if (sqrt(v[0]) < c->tol) {
      c->done = 1;
      c->status = PDEB200_OK;
    } else if (c->iter >= c->max_iter) {
      c->done = 1;
      c->status = PDEB200_ERR_NOT_CONVERGED;
    } else {
      c->beta = v[0] / c->rz;
      c->rz = v[0];
    }
  }
};

struct PostBeta {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->beta = v[0] / c->rz;
    c->rz = v[0];
  }
};

struct PostRZ {
  Ctl* c;
  __device__ void operator()(const double* v) const { c->rz = v[0]; }
};

// r.z summed by the last two colour passes of a V-cycle (k_rbgs DOT): the
// first stores its colour's part, the second adds its own and forms beta
constexpr int kAuxRzPart = 7;
struct PostRZPart {
  Ctl* c;
  __device__ void operator()(const double* v) const { c->aux[kAuxRzPart] = v[0]; }
};
struct PostBetaSplit {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    const double rz = c->aux[kAuxRzPart] + v[0];
    c->beta = rz / c->rz;
    c->rz = rz;
  }
};

// |b|^2 of the relative rule: tol2 = tol^2 |b|^2, immediate exit for b = 0
struct PostBB {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->bb = v[0];
    c->rr = v[0];
    c->tol2 = c->tol * c->tol * v[0];
    if (v[0] == 0.0) {
      c->done = 1;
      c->status = PDEB200_OK;
    }
  }
};

// initial |r|^2 of the reference CG: exit when sqrt(rr) < tol before iterating
struct PostRR0Ref {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->rr = v[0];
    c->rz = v[0];
    if (sqrt(v[0]) < c->tol) {
      c->done = 1;
      c->status = PDEB200_OK;
    }
  }
};

// relaxation: max|du| < tol stops sweeping (relaxation.cpp:557, solver.cpp:976)
struct PostDelta {
  Ctl* c;
  __device__ void operator()(const double* v) const {
    c->delta = v[0];
    c->iter += 1;
    if (v[0] < c->tol) {
      c->stop = 1;
      c->status = PDEB200_OK;
    } else if (c->iter >= c->max_iter) {
      c->stop = 1;
      c->status = PDEB200_ERR_NOT_CONVERGED;
    }
  }
};

// ------------------------------------------------------------- utilities

inline void ctl_init(Context* ctx, int max_iter, double tol, double brk) {
  std::memset(ctx->h_ctl, 0, sizeof(Ctl));
  ctx->h_ctl->max_iter = max_iter;
  ctx->h_ctl->tol = tol;
  ctx->h_ctl->brk = brk;
  ctx->h_ctl->status = PDEB200_ERR_NOT_CONVERGED;
  PDEB_CUDA(cudaMemcpyAsync(ctx->d_ctl, ctx->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
}

inline const Ctl& ctl_poll(Context* ctx) {
  PDEB_CUDA(cudaMemcpyAsync(ctx->h_ctl, ctx->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
  return *ctx->h_ctl;
}

inline void ctl_set_done(Context* ctx, int status) {
  int v[3] = {1, 1, status};
  PDEB_CUDA(cudaMemcpyAsync(ctx->d_ctl, v, sizeof(v), cudaMemcpyHostToDevice, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
}

// Enqueue iterations in growing batches and poll; `iterate()` enqueues one
// iteration. Returns when the device reports done/stop or the cancel flag is set.
// predict: the iterations monitor |r|^2 against tol2 (relative rule); after two
// polls the next batch is the number of iterations the observed reduction
// rate still needs, so few iterations are enqueued past convergence (they
// would return at once, but each still costs its launches).
template <class It>
pdeb200_status drive(Context* ctx, const pdeb200_options* o, int max_iter, It&& iterate, bool use_stop,
                     bool predict = false) {
  int enq = 0;
  int batch = 1;
  const int cap = o->check_interval > 0 ? o->check_interval : 16;
  double rr_prev = -1.0;
  int it_prev = 0;
  while (true) {
    for (int b = 0; b < batch && enq < max_iter; ++b, ++enq) iterate(enq);
    const Ctl& c = ctl_poll(ctx);
    if (c.done || (use_stop && c.stop)) return (pdeb200_status)c.status;
    if (enq >= max_iter) return PDEB200_ERR_NOT_CONVERGED;
    if (o->cancel && *o->cancel) {
      ctl_set_done(ctx, PDEB200_ERR_CANCELLED);
      return PDEB200_ERR_CANCELLED;
    }
    int next = batch * 2 < cap ? batch * 2 : cap;
    if (predict && c.rr > 0.0 && c.tol2 > 0.0) {
      if (rr_prev > 0.0 && c.iter > it_prev && c.rr < rr_prev) {
        const double rate = std::log(c.rr / rr_prev) / double(c.iter - it_prev);  // < 0
        const double need = std::log(c.tol2 / c.rr) / rate;
        if (need > 0.0 && need < double(cap)) next = std::max(1, (int)std::ceil(need));
      }
      rr_prev = c.rr;
      it_prev = c.iter;
    }
    batch = next;
  }
}

// One solver iteration captured once as a CUDA graph and replayed. `iterate`
// must only enqueue kernels on ctx->stream (they all read the device control
// block, so a replay after convergence is a no-op like a direct launch). The
// capture runs on the context's own stream, since the caller's stream may be
// the legacy default stream, which cannot be captured; replays go to
// ctx->stream. Off while per-kernel profiling is on or PDEB200_NO_GRAPH is set.
struct IterGraph {
  cudaGraphExec_t exec = nullptr;
  long long launches_per_iter = 0;
  IterGraph() = default;
  IterGraph(const IterGraph&) = delete;
  IterGraph& operator=(const IterGraph&) = delete;
  ~IterGraph() {
    if (exec) cudaGraphExecDestroy(exec);
  }
  template <class It>
  bool capture(Context* ctx, It&& iterate) {
    if (ctx->prof || std::getenv("PDEB200_NO_GRAPH") != nullptr) return false;
    cudaStream_t saved = ctx->stream;
    const long long before = ctx->launches;
    ctx->stream = ctx->own_stream;
    if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      ctx->stream = saved;
      cudaGetLastError();
      return false;
    }
    cudaGraph_t g = nullptr;
    try {
      iterate(0);
    } catch (...) {
      cudaStreamEndCapture(ctx->stream, &g);
      if (g) cudaGraphDestroy(g);
      ctx->stream = saved;
      cudaGetLastError();
      throw;
    }
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->stream = saved;
    launches_per_iter = ctx->launches - before;
    ctx->launches = before;
    if (e != cudaSuccess || !g) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return false;
    }
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      exec = nullptr;
      cudaGetLastError();
      return false;
    }
    return true;
  }
  void launch(Context* ctx) {
    PDEB_CUDA(cudaGraphLaunch(exec, ctx->stream));
    ctx->launches += launches_per_iter;
  }
};

inline void fill_boundary(Context* ctx, const GridDev& g, double* u, const Ctl* ctl, bool dirichlet_last = true) {
  const long long faces = 2LL * g.ny * g.nz + 2LL * g.nx * g.nz + (g.dim == 3 ? 2LL * g.nx * g.ny : 0);
  const int blocks = vec_blocks(faces, ctx);
  k_fill_boundary<<<blocks, 256, 0, ctx->stream>>>(g, u, ctl, dirichlet_last ? 1 : 0);
  ctx->count();
}

template <typename T>
void vfill(Context* ctx, long long n, T* p, T v, const Ctl* ctl) {
  k_fill<T><<<vec_blocks(n, ctx), 256, 0, ctx->stream>>>(n, p, v, ctl);
  ctx->count();
}


// ------------------------------------------------------------ rhs builders

// BuildRhs2D (src/backends/cpu/solver.cpp:167-232), any dimension: Dirichlet
// values on boundary nodes (last Dirichlet face written wins, 0 elsewhere),
// -f in the interior.
__global__ void k_full_rhs(GridDev g, const double* __restrict__ f, double f_const, double* __restrict__ b);

inline void build_full_rhs(Context* ctx, DevProblem& P, double* b) {
  k_full_rhs<<<vec_blocks(P.g.n, ctx), 256, 0, ctx->stream>>>(P.g, P.f, P.f_const, b);
  ctx->count();
}

template <class Coef>
void build_folded_rhs(Context* ctx, DevProblem& P, const Coef& cf, double* b) {
  PDEB_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * P.g.n, ctx->stream));
  k_folded_rhs<Coef><<<stencil_grid(P.g), stencil_block(), 0, ctx->stream>>>(P.g, cf, P.f, P.f_const, b);
  ctx->count();
}

// sum over all nodes of (b - L x)^2 with identity boundary rows
template <class Coef, class Post>
__global__ void __launch_bounds__(kBx* kBy) k_residual_full(GridDev g, Coef cf, const double* __restrict__ x,
                                                            const double* __restrict__ b, RedSlot slot, Post post) {
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
        const double zp = g.dim == 3 ? x[id + g.sxy] : 0.0;
        const double zm = g.dim == 3 ? x[id - g.sxy] : 0.0;
        v = s.c * x[id] + nb_sum<double>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, g.dim);
      }
      const double r = b[id] - v;
      acc[0] += r * r;
    }
  }
  grid_reduce<1, false>(acc, slot, post);
}

template <class Coef>
void full_residual_report(Context* ctx, DevProblem& P, const Coef& cf, const double* b, const double* x, double*,
                          pdeb200_report* rep) {
  if (!rep) return;
  const long long n = P.g.n;
  k_residual_full<Coef, PostStoreRR><<<stencil_grid_full(P.g), stencil_block(), 0, ctx->stream>>>(
      P.g, cf, x, b, ctx->slot(), PostStoreRR{ctx->d_ctl});
  k_dot<double, PostBBOnly><<<vec_blocks(n, ctx), 256, 0, ctx->stream>>>(n, b, b, ctx->slot(1),
                                                                       PostBBOnly{ctx->d_ctl}, nullptr);
  ctx->count(2);
  const Ctl& c = ctl_poll(ctx);
  rep->residual_l2 = std::sqrt(c.rr);
  rep->rhs_l2 = std::sqrt(c.bb);
  rep->rel_residual = c.bb > 0 ? rep->residual_l2 / rep->rhs_l2 : 0.0;
}

template <class Coef>
void folded_residual_report(Context* ctx, DevProblem& P, const Coef& cf, const double* bf, const double* x,
                            double* scratch, pdeb200_report* rep) {
  if (!rep) return;
  const long long n = P.g.n;
  k_residual_folded<Coef, double, double, 1, PostStoreRR><<<stencil_grid(P.g), stencil_block(), 0, ctx->stream>>>(
      P.g, cf, x, bf, scratch, ctx->slot(), PostStoreRR{ctx->d_ctl}, nullptr);
  k_dot<double, PostBBOnly><<<vec_blocks(n, ctx), 256, 0, ctx->stream>>>(n, bf, bf, ctx->slot(1),
                                                                        PostBBOnly{ctx->d_ctl}, nullptr);
  ctx->count(2);
  const Ctl& c = ctl_poll(ctx);
  rep->residual_l2 = std::sqrt(c.rr);
  rep->rhs_l2 = std::sqrt(c.bb);
  rep->rel_residual = c.bb > 0 ? rep->residual_l2 / rep->rhs_l2 : 0.0;
}

// ------------------------------------------------------------ MG hierarchy

// Coarsening of the B200 hierarchy, per dimension: a dimension with >= 5 nodes
// coarsens to ceil((n-1)/2)+1 nodes (2:1 and nested for odd n) when its
// spacing is below twice the smallest spacing of the grid; others keep their
// size (semi-coarsening keeps the coarse cells near isotropic on elongated
// domains). Returns false when no dimension coarsens.
inline int coarse_size(int n) { return n / 2 + 1; }  // ceil((n-1)/2) + 1

inline bool coarse_dims(const GridDev& g, const pdeb200_problem* hp, int nc[3]) {
  const int n[3] = {g.nx, g.ny, g.nz};
  const double len[3] = {hp->xmax - hp->xmin, hp->ymax - hp->ymin, hp->zmax - hp->zmin};
  const int dims = g.dim == 3 ? 3 : 2;
  double h[3], hmin = 0.0;
  for (int d = 0; d < dims; ++d) {
    h[d] = len[d] / double(n[d] - 1);
    if (d == 0 || h[d] < hmin) hmin = h[d];
  }
  bool any = false;
  for (int d = 0; d < 3; ++d) {
    nc[d] = n[d];
    if (d < dims && n[d] >= 5 && h[d] < 2.0 * hmin) {
      nc[d] = coarse_size(n[d]);
      any = true;
    }
  }
  return any;
}

// the z map of a level pair is the identity or nested 2:1 (host-side test of
// z_marchable in kernels.cuh)
inline bool z_nested(const GridDev& gf, const GridDev& gc) {
  return gf.dim != 3 || gc.nz == gf.nz || 2 * gc.nz - 1 == gf.nz;
}

// a 3D level pair nested 2:1 in every dimension (k_prolong_pair)
inline bool nested_3d(const GridDev& gf, const GridDev& gc) {
  return gf.dim == 3 && 2 * gc.nx - 1 == gf.nx && 2 * gc.ny - 1 == gf.ny && 2 * gc.nz - 1 == gf.nz;
}

// launch shape of k_prolong_pair: 32 x 8 coarse columns per block, coarse-plane
// chunks for about 148 x 14 blocks (32 chunks into 129^3 coarse: 68 us at
// 257^3 fine, against 72 / 84 us with 16 / 8 chunks and 70 us with 64)
inline dim3 prolong_pair_grid(const GridDev& gc) {
  const dim3 xy((gc.nx - 1 + kBx - 1) / kBx, (gc.ny - 1 + kBy - 1) / kBy, 1);
  const long long xyb = (long long)xy.x * xy.y;
  long long chunks = (148LL * 14 + xyb - 1) / xyb;
  if (chunks > gc.nz - 1) chunks = gc.nz - 1;
  if (chunks > kMaxGridBlocks / xyb) chunks = kMaxGridBlocks / xyb;
  if (chunks < 1) chunks = 1;
  return dim3(xy.x, xy.y, (unsigned)chunks);
}

template <typename KT>
inline void inject_k(Context* ctx, const GridDev& gf, const GridDev& gc, const KT* kf, KT* kc) {
  k_inject<KT><<<vec_blocks(gc.n, ctx), 256, 0, ctx->stream>>>(gf, gc, kf, kc);
  ctx->count();
}

// Coarse coefficients: constants are re-evaluated with the coarse spacing,
// sampled fields are injected (k_c(I) = k_f(2I)).
// Coarse constant stencils are rediscretised at the coarse spacing. With
// convection, the coarse diffusion is raised where needed so the coarse cell
// Peclet number |c| H / (2|a|) stays <= 1 (central differences keep a
// diagonally dominant coarse operator); the fine operator is never modified.
inline CoefConst coarsen_coef(Context*, const DevProblem& P, const CoefConst&, const GridDev&, const GridDev& gc,
                              double dx, double dy, double dz, std::vector<Buf>*) {
  auto stab = [](double a, double c, double h) {
    const double need = std::fabs(c) * h * 0.5;
    return (a <= 0.0 && -a < need) ? -need : a;
  };
  return make_const(stab(P.a, P.c, dx), stab(P.b, P.d, dy), gc.dim == 3 ? stab(P.az, P.dzc, dz) : P.az, P.c, P.d,
                    P.dzc, P.e, dx, dy, dz, gc.dim);
}

template <typename KT>
inline CoefDivk<KT> coarsen_coef(Context* ctx, const DevProblem& P, const CoefDivk<KT>& f, const GridDev& gf,
                                 const GridDev& gc, double dx, double dy, double dz, std::vector<Buf>* owned) {
  CoefDivk<KT> c = f;
  owned->emplace_back(sizeof(KT) * gc.n, ctx->stream);
  KT* kc = owned->back().template as<KT>();
  inject_k<KT>(ctx, gf, gc, f.k, kc);
  c.k = kc;
  c.ihx2 = 1.0 / (dx * dx);
  c.ihy2 = 1.0 / (dy * dy);
  c.ihz2 = gc.dim == 3 ? 1.0 / (dz * dz) : 0.0;
  c.cx = P.c / (2.0 * dx);
  c.dyc = P.d / (2.0 * dy);
  c.dzc = gc.dim == 3 ? P.dzc / (2.0 * dz) : 0.0;
  return c;
}

inline CoefNodal coarsen_coef(Context* ctx, const DevProblem&, const CoefNodal& f, const GridDev& gf,
                              const GridDev& gc, double dx, double dy, double dz, std::vector<Buf>* owned) {
  CoefNodal c = f;
  owned->emplace_back(sizeof(double) * 7 * gc.n, ctx->stream);
  double* dst = owned->back().as<double>();
  for (int q = 0; q < 7; ++q) inject_k<double>(ctx, gf, gc, f.nodal + (long long)q * f.n, dst + (long long)q * gc.n);
  c.nodal = dst;
  c.n = gc.n;
  c.dx2 = dx * dx;
  c.dy2 = dy * dy;
  c.dz2 = dz * dz;
  c.tdx = 2.0 * dx;
  c.tdy = 2.0 * dy;
  c.tdz = 2.0 * dz;
  return c;
}

// Geometric hierarchy of the folded operator. Coarsening per coarse_dims
// (odd cubes nest 2:1 as in the reference's multigrid.cpp:150-170, continued
// down to 3 nodes; even sizes use the non-nested maps of kernels.cuh); face
// closures are rediscretised with the coarse spacing.
// Each level has two field buffers: smoothing sweeps are fused red-black
// passes that read one buffer and write the other.
template <class Coef, typename T>
struct Hierarchy {
  struct Level {
    GridDev g;
    Coef cf;
    T* xa;   // written by the first sweep from zero
    T* xb;
    T* b;
    T* r;
    T* out;  // buffer holding this level's result after a V-cycle
    bool single_pass = false;  // sweeps by k_rbgs_sweep (x_in -> x_out) instead of colour passes
    bool march = false;        // sweeps by k_rbgs_march (x_in -> x_out) instead of colour passes
  };
  // With PDEB200_STAGED_SWEEP set, levels with at least this many nodes use
  // the staged single-pass sweep (FP64 constant or divergence-form
  // coefficients). It moves half the DRAM bytes of two colour passes but on
  // B200 it is issue- and barrier-bound and about 10% slower at 257^3, so the
  // colour passes stay the default.
  static constexpr long long kSweepMinNodes = 1LL << 18;
  // With PDEB200_MARCH set, levels of at least kMarchMinNodes nodes (3D,
  // FP64, constant or divergence-form coefficients) smooth with the
  // single-pass marching sweep (k_rbgs_march). It moves 552 MB per sweep at
  // 257^3 against 2 x 512 MB for two colour passes, but it is latency- and
  // barrier-bound (about 21 warps per SM, one barrier per plane): 255 against
  // 226 us per sweep on a box where a colour pass takes 113 us, so the colour
  // passes stay the default.
  static constexpr long long kMarchMinNodes = 1LL << 18;
  static constexpr bool kSweepCoef =
      std::is_same<T, double>::value &&
      (std::is_same<Coef, CoefConst>::value || std::is_same<Coef, CoefDivk<double>>::value);
  std::vector<Level> levels;
  std::vector<Buf> owned;
  int pre = 2, post = 2, coarse_iters = 50;
  bool needs_fold = false;  // some face is Neumann/Robin

  T* alloc(Context* ctx, long long n) {
    owned.emplace_back(sizeof(T) * n, ctx->stream);
    T* p = owned.back().template as<T>();
    PDEB_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * n, ctx->stream));
    return p;
  }

  // Levels from tail_l0 down run as one single-block launch (k_tail_vcycle).
  static constexpr long long kTailMaxNodes = 1100;
  int tail_l0 = -1;
  TailLevel<Coef, T>* d_tail = nullptr;

  bool coarse_in_smem(const Level& L) const {
    const long long interior = (long long)(L.g.nx - 2) * (L.g.ny - 2) * (L.g.dim == 3 ? L.g.nz - 2 : 1);
    return L.g.n <= kCoarseMaxNodes && interior <= kCoarseMaxInterior;
  }

  void build(Context* ctx, DevProblem& P, const pdeb200_problem* hp, const Coef& cf0, const pdeb200_options* o) {
    fused = std::getenv("PDEB200_FUSED_SWEEP") != nullptr;
    needs_fold = false;
    for (int f = 0; f < 6; ++f)
      if (P.g.face[f].active && P.g.face[f].kind != kDirichlet) needs_fold = true;
    pre = o->mg_pre_smooth > 0 ? o->mg_pre_smooth : 0;
    post = o->mg_post_smooth > 0 ? o->mg_post_smooth : 0;
    coarse_iters = o->mg_coarse_iters > 1 ? o->mg_coarse_iters : 1;
    const int max_levels = o->mg_max_levels > 1 ? o->mg_max_levels : 1;
    Level l0;
    l0.g = P.g;
    l0.cf = cf0;
    l0.xa = alloc(ctx, P.g.n);
    l0.xb = alloc(ctx, P.g.n);
    l0.b = nullptr;
    l0.r = alloc(ctx, P.g.n);
    levels.push_back(l0);
    int stride = 1;
    int nc[3];
    while ((int)levels.size() < max_levels && coarse_dims(levels.back().g, hp, nc)) {
      const GridDev& gf = levels.back().g;
      Level c;
      c.g = gf;
      c.g.nx = nc[0];
      c.g.ny = nc[1];
      c.g.nz = gf.dim == 3 ? nc[2] : 1;
      c.g.sxy = (long long)c.g.nx * c.g.ny;
      c.g.n = c.g.sxy * c.g.nz;
      stride *= 2;
      const double cdx = (hp->xmax - hp->xmin) / (double)(c.g.nx - 1);
      const double cdy = (hp->ymax - hp->ymin) / (double)(c.g.ny - 1);
      const double cdz = gf.dim == 3 ? (hp->zmax - hp->zmin) / (double)(c.g.nz - 1) : 0.0;
      build_faces(ctx, hp, c.g.nx, c.g.ny, c.g.nz, cdx, cdy, cdz, stride, &c.g, &owned);
      c.cf = coarsen_coef(ctx, P, levels.back().cf, gf, c.g, cdx, cdy, cdz, &owned);
      c.xa = alloc(ctx, c.g.n);
      c.xb = alloc(ctx, c.g.n);
      c.b = alloc(ctx, c.g.n);
      c.r = alloc(ctx, c.g.n);
      levels.push_back(c);
    }
    // single-block tail: the first level small enough, with at most
    // kTailMaxLevels levels below it (colour-pass form only)
    tail_l0 = -1;
    if (!fused && std::getenv("PDEB200_NO_TAIL") == nullptr) {
      for (size_t l = 0; l < levels.size(); ++l)
        if (levels[l].g.n <= kTailMaxNodes && (int)(levels.size() - l) <= kTailMaxLevels) {
          tail_l0 = (int)l;
          break;
        }
    }
    if (tail_l0 >= 0) {
      std::vector<TailLevel<Coef, T>> tl;
      for (size_t l = tail_l0; l < levels.size(); ++l)
        tl.push_back(TailLevel<Coef, T>{levels[l].g, levels[l].cf, levels[l].xa, levels[l].b, levels[l].r});
      owned.emplace_back(sizeof(TailLevel<Coef, T>) * tl.size(), ctx->stream);
      d_tail = owned.back().template as<TailLevel<Coef, T>>();
      PDEB_CUDA(cudaMemcpyAsync(d_tail, tl.data(), sizeof(TailLevel<Coef, T>) * tl.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
      PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    // result buffer of each level after a V-cycle (fixed, so launches can be captured):
    // the first sweep from zero writes xa, every later sweep flips the buffer
    const bool sweep_env = std::getenv("PDEB200_STAGED_SWEEP") != nullptr;
    const bool march_env = std::getenv("PDEB200_MARCH") != nullptr;
    for (size_t l = 0; l < levels.size(); ++l) {
      Level& L = levels[l];
      L.single_pass = kSweepCoef && sweep_env && !fused && l + 1 < levels.size() && L.g.dim == 3 &&
                      L.g.n >= kSweepMinNodes;
      L.march = kSweepCoef && march_env && !fused && !L.single_pass && l + 1 < levels.size() && L.g.dim == 3 &&
                L.g.n >= kMarchMinNodes;
      if (!fused && !L.single_pass && !L.march) {
        L.out = L.xa;
        continue;
      }
      int flips;
      if (l + 1 == levels.size())
        flips = coarse_in_smem(L) ? 0 : coarse_iters - 1;
      else
        flips = pre > 0 ? pre - 1 + post : post;
      L.out = (flips & 1) ? L.xb : L.xa;
    }
  }

  // `sweeps` red-black sweeps starting from `cur` (or from zero); returns the
  // buffer holding the result. Two forms with identical arithmetic: colour
  // passes in place (default), or fused single-pass sweeps that read one
  // buffer and write the other.
  bool fused = false;
  T* sweeps_from(Context* ctx, Level& L, const T* b, T* cur, int sweeps, int first, bool from_zero,
                 const Ctl* ctl, int lvl, const RedSlot* dot_last = nullptr) {
    const dim3 grid = rbgs_grid(L.g), block = stencil_block();
    const dim3 zgrid = stencil_grid_auto(L.g);  // the pass from zero (fewer registers) keeps the default
    const double dofs = interior_dofs(L.g);
    if constexpr (kSweepCoef) {
      if (L.march) {
        constexpr size_t smem = march_smem_bytes<Coef>();
        static bool attr_set[64] = {false};
        const int dv = ctx->dev >= 0 && ctx->dev < 64 ? ctx->dev : 0;
        if (!attr_set[dv]) {
          PDEB_CUDA(cudaFuncSetAttribute(k_rbgs_march<Coef, false, NoPost>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          PDEB_CUDA(cudaFuncSetAttribute(k_rbgs_march<Coef, true, PostBeta>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
          attr_set[dv] = true;
        }
        const dim3 mgrid = march_grid(L.g);
        for (int s = 0; s < sweeps; ++s) {
          const bool zero = from_zero && s == 0;
          T* in = zero ? L.xb : cur;
          T* out = zero ? L.xa : (cur == L.xa ? L.xb : L.xa);
          // x read and written once, b and k read once: 32 B per DOF (24 from zero)
          ProfScope ps(ctx, zero ? "march_sweep_zero" : "march_sweep", lvl, dofs * (zero ? 3.0 : 4.0) * sizeof(T));
          if (dot_last && s + 1 == sweeps)
            k_rbgs_march<Coef, true, PostBeta><<<mgrid, kMThreads, smem, ctx->stream>>>(
                L.g, L.cf, b, in, out, first, zero ? 1 : 0, ctl, *dot_last, PostBeta{const_cast<Ctl*>(ctl)});
          else
            k_rbgs_march<Coef><<<mgrid, kMThreads, smem, ctx->stream>>>(L.g, L.cf, b, in, out, first, zero ? 1 : 0,
                                                                         ctl);
          ctx->count();
          cur = out;
        }
        return cur;
      }
      if (L.single_pass) {
        // per instantiation and device, before its first launch there
        static bool attr_set[64] = {false};
        const int dv = ctx->dev >= 0 && ctx->dev < 64 ? ctx->dev : 0;
        if (!attr_set[dv]) {
          PDEB_CUDA(cudaFuncSetAttribute(k_rbgs_sweep<Coef>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSwSmemBytes));
          attr_set[dv] = true;
        }
        const dim3 sgrid = sweep_grid(L.g);
        for (int s = 0; s < sweeps; ++s) {
          const bool zero = from_zero && s == 0;
          T* in = zero ? L.xb : cur;
          T* out = zero ? L.xa : (cur == L.xa ? L.xb : L.xa);
          {
            // x read and written once, b and k read once: 32 B per DOF
            ProfScope ps(ctx, "rbgs_sweep", lvl, dofs * 4.0 * sizeof(T));
            k_rbgs_sweep<Coef><<<sgrid, kSwThreads, kSwSmemBytes, ctx->stream>>>(L.g, L.cf, b, in, out, first,
                                                                                 zero ? 1 : 0, ctl);
          }
          ctx->count();
          cur = out;
        }
        return cur;
      }
    }
    if (!fused) {
      // in place: the buffer never changes; flips are bookkeeping only. From
      // zero, the first pass reads no field values (k_rbgs ZERO) and the
      // field is not cleared; without sweeps it is cleared.
      if (from_zero) {
        cur = L.xa;
        if (sweeps == 0) {
          ProfScope ps(ctx, "zero_fill", lvl, dofs * sizeof(T));
          vfill<T>(ctx, L.g.n, L.xa, T(0), ctl);
        }
      }
      for (int s = 0; s < sweeps; ++s) {
        for (int half = 0; half < 2; ++half) {
          if (from_zero && s == 0 && half == 0) {
            // b and the written half of x: 8 B per DOF in FP64
            ProfScope ps(ctx, "rbgs_zero_pass", lvl, dofs * sizeof(T));
            launch_dep(ctx, zgrid, block, 0, k_rbgs<Coef, T, T, true>, L.g, L.cf, b, cur, first, ctl, RedSlot{},
                       NoPost{});
            continue;
          }
          ProfScope ps(ctx, "rbgs_color_pass", lvl, dofs * 2.0 * sizeof(T));
          launch_dep(ctx, grid, block, 0, k_rbgs<Coef, T, T>, L.g, L.cf, b, cur, first ^ half, ctl, RedSlot{},
                     NoPost{});
        }
        ctx->count(2);
      }
      return cur;
    }
    const dim3 fgrid = fused_grid(L.g);
    for (int s = 0; s < sweeps; ++s) {
      const bool zero = from_zero && s == 0;
      T* in = zero ? L.xb : cur;
      T* out = zero ? L.xa : (cur == L.xa ? L.xb : L.xa);
      {
        ProfScope ps(ctx, "rbgs_sweep", lvl, dofs * 4.0 * sizeof(T));
        k_rbgs_fused<Coef, T, T><<<fgrid, block, 0, ctx->stream>>>(L.g, L.cf, b, in, out, first, zero ? 1 : 0, ctl);
      }
      ctx->count();
      cur = out;
    }
    return cur;
  }

  void level(Context* ctx, int l, const T* rhs0, const Ctl* ctl) {
    Level& L = levels[l];
    const T* b = l == 0 ? rhs0 : L.b;
    const double dofs = interior_dofs(L.g);
    if (l == tail_l0) {
      ProfScope ps(ctx, "tail_vcycle", l, 0.0);
      launch_dep(ctx, dim3(1), dim3(kTailThreads), 0, k_tail_vcycle<Coef, T>, (const TailLevel<Coef, T>*)d_tail,
                 (int)levels.size() - l, b, pre, post, coarse_iters, needs_fold ? 1 : 0, ctl);
      ctx->count();
      return;
    }
    if (l == (int)levels.size() - 1) {
      if (coarse_in_smem(L)) {
        ProfScope ps(ctx, "coarse_solve", l, 0.0);
        k_coarse_solve_smem<Coef, T, T><<<1, 256, 0, ctx->stream>>>(L.g, L.cf, b, L.xa, coarse_iters, ctl);
        ctx->count();
      } else {
        T* cur = sweeps_from(ctx, L, b, L.xa, coarse_iters, 0, true, ctl, l);
        (void)cur;
      }
      return;
    }
    T* cur = L.xa;
    if (pre > 0) {
      cur = sweeps_from(ctx, L, b, L.xa, pre, 0, true, ctl, l);
    } else {
      vfill<T>(ctx, L.g.n, L.xa, T(0), ctl);
    }
    {
      ProfScope ps(ctx, "residual", l, dofs * 4.0 * sizeof(T));
      // levels that fit in L2: 148 x 6 target blocks (65^3: 4.6 -> 3.7 us per
      // launch in a replayed graph; 129^3 unchanged); larger levels 148 x 24
      // (12 z chunks at 257^3, an even number of planes per chunk for the
      // two-plane trips: 108.7 -> 103.6 us per launch in the solve)
      launch_dep(ctx, stencil_grid_auto(L.g, L.g.n > (1LL << 22) ? 148 * 24 : 148 * 6), stencil_block(), 0,
                 k_residual_folded<Coef, T, T, 0, NoPost>, L.g, L.cf, (const T*)cur, b, L.r, RedSlot{}, NoPost{},
                 ctl);
    }
    Level& C = levels[l + 1];
    {
      ProfScope ps(ctx, "restrict", l, dofs * sizeof(T) * (1.0 + 1.0 / (L.g.dim == 3 ? 8.0 : 4.0)));
      if (z_nested(L.g, C.g))
        // 4 coarse planes per thread share plane sums on large levels (into
        // 129^3: 58.3 us, against 61.3 with 8 and 76.0 with 16); small levels
        // take one plane per thread (latency rather than bytes). The result
        // does not depend on the chunking: a chunk's first plane sum is
        // recomputed with the same arithmetic as a carried one.
        launch_dep(ctx, stencil_grid_full(C.g, C.g.n > (1LL << 20) ? 4 : 1), stencil_block(), 0,
                   k_restrict_march<T, T>, L.g, C.g, (const T*)L.r, C.b, ctl);
      else
        launch_dep(ctx, stencil_grid_full(C.g, 1), stencil_block(), 0, k_restrict_fw<T, T>, L.g, C.g, (const T*)L.r,
                   C.b, ctl);
    }
    if (needs_fold) {
      ProfScope ps(ctx, "restrict_fold", l, 0.0);
      const FoldLayers lay = fold_layers(C.g);
      const int blocks = (int)std::max<long long>(1, std::min<long long>((lay.start[6] + 255) / 256, 148LL * 16));
      launch_dep(ctx, dim3(blocks), dim3(256), 0, k_restrict_fold_faces<T>, C.g, lay, C.b, ctl);
      ctx->count();
    }
    ctx->count(2);
    level(ctx, l + 1, rhs0, ctl);
    {
      ProfScope ps(ctx, "prolong_add", l, dofs * sizeof(T) * (2.0 + 1.0 / (L.g.dim == 3 ? 8.0 : 4.0)));
      if (nested_3d(L.g, C.g))
        launch_dep(ctx, prolong_pair_grid(C.g), stencil_block(), 0, k_prolong_pair<T, T>, L.g, C.g, (const T*)C.out,
                   cur, ctl);
      else if (z_nested(L.g, C.g))
        // 148*24 target blocks (12 z chunks at 257^3): 101.7 -> 97 us against
        // 148*16; 148*12 and 148*40 are slower
        launch_dep(ctx, stencil_grid_auto(L.g, 148 * 24), stencil_block(), 0, k_prolong_march<T, T>, L.g, C.g,
                   (const T*)C.out, cur, ctl);
      else
        launch_dep(ctx, stencil_grid_auto(L.g), stencil_block(), 0, k_prolong_add<T, T>, L.g, C.g, (const T*)C.out,
                   cur, ctl);
    }
    ctx->count();
    if (l == 0 && dot_slot && post > 0 && L.march) {
      // the last sweep also sums r.z (b is r on level 0) and forms beta
      cur = sweeps_from(ctx, L, b, cur, post, 1, false, ctl, l, dot_slot);
      dot_done = true;
    } else if (l == 0 && dot_slot && post > 0 && !fused && !L.single_pass) {
      // the last sweep's two passes also sum r.z (b is r on level 0)
      cur = sweeps_from(ctx, L, b, cur, post - 1, 1, false, ctl, l);
      const dim3 grid = rbgs_grid(L.g), block = stencil_block();
      {
        ProfScope ps(ctx, "rbgs_color_pass", l, dofs * 2.0 * sizeof(T));
        launch_dep(ctx, grid, block, 0, k_rbgs<Coef, T, T, false, true, PostRZPart>, L.g, L.cf, b, cur, 1, ctl,
                   *dot_slot, PostRZPart{const_cast<Ctl*>(ctl)});
      }
      {
        ProfScope ps(ctx, "rbgs_color_pass", l, dofs * 2.0 * sizeof(T));
        launch_dep(ctx, grid, block, 0, k_rbgs<Coef, T, T, false, true, PostBetaSplit>, L.g, L.cf, b, cur, 0, ctl,
                   *dot_slot, PostBetaSplit{const_cast<Ctl*>(ctl)});
      }
      ctx->count(2);
      dot_done = true;
    } else {
      cur = sweeps_from(ctx, L, b, cur, post, 1, false, ctl, l);
    }
  }

  // z = M rhs0; the result is in levels[0].out
  void vcycle(Context* ctx, const T* rhs0, const Ctl* ctl) {
    dot_slot = nullptr;
    level(ctx, 0, rhs0, ctl);
  }
  // z = M r and, when the finest level's last sweep could carry it, beta of
  // preconditioned CG from r.z (PostBetaSplit). Returns false when the caller
  // must compute r.z itself.
  bool vcycle_dot(Context* ctx, const T* r, const Ctl* ctl, const RedSlot& slot) {
    dot_slot = &slot;
    dot_done = false;
    level(ctx, 0, r, ctl);
    dot_slot = nullptr;
    return dot_done;
  }
  const RedSlot* dot_slot = nullptr;
  bool dot_done = false;
  T* z() const { return levels[0].out; }
};

// -------------------------------------------------- drivers in other units

template <class Coef>
pdeb200_status gauss_seidel(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_out,
                            pdeb200_report* rep);
template <class Coef>
pdeb200_status bicgstab_reference(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o,
                                  double* d_x, pdeb200_report* rep);
template <class Coef>
pdeb200_status gmres_reference(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_options* o, double* d_x,
                               pdeb200_report* rep);
pdeb200_status mg_vcycle_reference(Context* ctx, DevProblem& P, const pdeb200_problem* hp, const pdeb200_options* o,
                                   double* d_out, pdeb200_report* rep);
template <class Coef>
pdeb200_status mixed_refinement(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_problem* hp,
                                const pdeb200_options* o, double* d_x, pdeb200_report* rep);
template <class Coef>
pdeb200_status mg_bicgstab(Context* ctx, DevProblem& P, const Coef& cf, const pdeb200_problem* hp,
                           const pdeb200_options* o, double* d_x, pdeb200_report* rep);

}  // namespace pdeb
