// Kernels of the batched solver. A batch is many independent grids ("members")
// of mixed sizes and dimensions solved together: every phase of the solver is
// ONE launch over a table of tiles that covers the matching level of every
// member, so a 33x33 grid and a 129^3 grid share each launch and the small
// grids no longer pay a launch per kernel.
//
// Per member the algorithm is FP32 MG-preconditioned CG inside FP64 iterative
// refinement (the precision form): the outer residual r = b - A x, the
// solution update, every inner product and the coarsest-grid solve are FP64;
// the MG V-cycle and the inner Krylov vectors are FP32 (hierarchy k in FP32 or
// BF16). Each member carries its own state machine (BMember::state) advanced
// by the reductions' post steps, so members converge independently and a
// finished member's tiles return at once.
//
// Tiles cover interior nodes only: tile T holds columns
// i in [1 + T.x0, 1 + T.x0 + T.w), j in [1 + T.y0, 1 + T.y0 + T.h) and planes
// k in [T.z0, T.z1). Kernels read the level and member descriptors straight
// from global memory (one L1 line broadcast to the block), so a block starts
// streaming its tile without a staging barrier.
// A member's coarsest level is one whole-grid tile (coarse = 1), solved by
// the block that restricts into it.
#pragma once

#include <type_traits>

#include "kernels.cuh"

namespace pdeb {

enum BState : int { kBDone = 0, kBNeedOuter = 1, kBInnerStart = 2, kBInnerRun = 3 };

// One level of one member.
struct BLevel {
  GridDev g;
  int kind;       // kConst / kDivk
  int member;
  int prev;       // finer level record (-1 on level 0)
  int next;       // coarser level record (-1 on the coarsest)
  int coarsest;
  int level;
  CoefConst cc;                                   // kConst stencil of this level
  double ihx2, ihy2, ihz2, cx, dyc, dzc, e;       // kDivk scalars of this level
  const void* kh;                                 // hierarchy k (float or bf16)
  float* x;                                       // correction (level 0: z = M r)
  float* b;                                       // right-hand side (level 0: PCG residual r)
  float* r;                                       // residual scratch
};

// Per-member solver state and level-0 vectors.
struct BMember {
  int state;
  int outer;        // outer residual evaluations so far
  int inner;        // inner iterations of the current refinement step
  int inner_total;
  int max_inner, max_outer;
  int tile0, ntiles;  // level-0 tiles [tile0, tile0 + ntiles)
  int first;          // the coming p update starts a new inner solve
  int status;
  int e_valid;        // e holds a correction not yet added to x
  int level0;
  unsigned ticket;
  int pad;
  double bb;        // |b|^2 (FP64)
  double rr0;       // |r|^2 at the start of the inner solve
  double rr;        // inner |r|^2
  double rr_outer;  // FP64 |b - A x|^2 at the last outer evaluation
  double rz, alpha, beta;
  double tol2;        // tol^2 (outer, relative to |b|)
  double tol2_inner;  // inner_tol^2 (relative to rr0)
  double tol2_step;   // this inner solve's target (relative to rr0): tol2_inner, or looser on a last step
  double* x64;
  double* b64;
  const double* f64;
  const double* k64;
  const float* k32;
  float* p;
  float* q;
  float* e;
};

struct alignas(16) BTile {
  int lev, member;
  int x0, y0;
  int z0, z1;
  unsigned short w, h;   // extent in nodes
  unsigned char lw;      // log2 of the padded row width (w <= 1 << lw)
  unsigned char coarse;  // whole-grid tile of a coarsest level
  unsigned char pad[2];
};

// Visits the (i,j) columns of tile T that this thread owns: thread t takes
// column t & (W-1) of row t >> lw (W = 1 << lw), so a warp covers 32
// consecutive nodes of a row.
template <class F>
__device__ __forceinline__ void tile_columns(const BTile& T, F&& f) {
  const int mask = (1 << T.lw) - 1;
  const int total = int(T.h) << T.lw;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int a = t & mask;
    if (a >= int(T.w)) continue;
    f(1 + T.x0 + a, 1 + T.y0 + (t >> T.lw));
  }
}

// Member fields written by the post steps are read with L2-coherent loads.
__device__ __forceinline__ int bstate(const BMember* m) { return __ldcg(&m->state); }
__device__ __forceinline__ bool vcycle_state(int s) { return s == kBInnerStart || s == kBInnerRun; }

// Folded stencil of interior node (i,j,kk) of level L with coefficient field k.
template <typename T, typename KT>
__device__ __forceinline__ Stencil<T> bstencil(const BLevel& L, const KT* k, int i, int j, int kk, long long id,
                                               double* shift) {
  Stencil<T> s;
  if (L.kind == kConst) {
    s = L.cc.template at<T>(L.g, id);
  } else {
    CoefDivk<KT> c;
    c.k = k;
    c.ihx2 = L.ihx2;
    c.ihy2 = L.ihy2;
    c.ihz2 = L.ihz2;
    c.cx = L.cx;
    c.dyc = L.dyc;
    c.dzc = L.dzc;
    c.e = L.e;
    s = c.template at<T>(L.g, id);
  }
  fold_faces<T>(L.g, i, j, kk, s, shift);
  return s;
}

// FP32 folded stencil of one level with its scalars in registers, loaded once
// per block (the level descriptor stays in global memory for the face data,
// read only at face-adjacent nodes). Indices are 32-bit offsets within the
// level's arrays (a member level has fewer than 2^31 nodes).
template <typename KT>
struct FStencil {
  int nx, ny, nz, dim, sxy, kind;
  float ihx2, ihy2, ihz2, cx, dyc, dzc, e;
  float c0, xm0, xp0, ym0, yp0, zm0, zp0;
  const KT* k;
  const GridDev* g;
  __device__ __forceinline__ void load(const BLevel& L, const KT* kk) {
    nx = L.g.nx;
    ny = L.g.ny;
    nz = L.g.nz;
    dim = L.g.dim;
    sxy = int(L.g.sxy);
    kind = L.kind;
    ihx2 = float(L.ihx2);
    ihy2 = float(L.ihy2);
    ihz2 = float(L.ihz2);
    cx = float(L.cx);
    dyc = float(L.dyc);
    dzc = float(L.dzc);
    e = float(L.e);
    c0 = float(L.cc.c);
    xm0 = float(L.cc.xm);
    xp0 = float(L.cc.xp);
    ym0 = float(L.cc.ym);
    yp0 = float(L.cc.yp);
    zm0 = float(L.cc.zm);
    zp0 = float(L.cc.zp);
    k = kk;
    g = &L.g;
  }
  __device__ __forceinline__ float kv(int id) const {
    if constexpr (sizeof(KT) == 2)
      return __bfloat162float(k[id]);
    else
      return __ldg(k + id);
  }
  // D: the grid dimension when the caller knows it at compile time, else 0
  template <int D = 0>
  __device__ __forceinline__ Stencil<float> at(int i, int j, int kz, int id) const {
    const bool d3 = D ? D == 3 : dim == 3;
    Stencil<float> s;
    if (kind == kConst) {
      s.c = c0;
      s.xm = xm0;
      s.xp = xp0;
      s.ym = ym0;
      s.yp = yp0;
      s.zm = zm0;
      s.zp = zp0;
    } else {
      const float kc = kv(id);
      const float kxm = 0.5f * (kc + kv(id - 1)), kxp = 0.5f * (kc + kv(id + 1));
      const float kym = 0.5f * (kc + kv(id - nx)), kyp = 0.5f * (kc + kv(id + nx));
      s.xm = -kxm * ihx2 - cx;
      s.xp = -kxp * ihx2 + cx;
      s.ym = -kym * ihy2 - dyc;
      s.yp = -kyp * ihy2 + dyc;
      float c = (kxm + kxp) * ihx2 + (kym + kyp) * ihy2;
      if (d3) {
        const float kzm = 0.5f * (kc + kv(id - sxy)), kzp = 0.5f * (kc + kv(id + sxy));
        s.zm = -kzm * ihz2 - dzc;
        s.zp = -kzp * ihz2 + dzc;
        c += (kzm + kzp) * ihz2;
      } else {
        s.zm = s.zp = 0.f;
      }
      s.c = c + e;
    }
    if (i == 1 || i == nx - 2 || j == 1 || j == ny - 2 || (d3 && (kz == 1 || kz == nz - 2)))
      fold_faces<float, D>(*g, i, j, kz, s, nullptr);
    return s;
  }
};

__device__ __forceinline__ long long bid(const GridDev& g, int i, int j, int k) {
  return ((long long)k * g.ny + j) * g.nx + i;
}

// Per-member reduction: every tile stores its block sum, the member's last
// tile (atomic ticket) adds the member's partials in tile order and runs
// post(member, sums). Deterministic for a given tiling, and independent of
// which other members share the launch.
template <int NV, class Post>
__device__ __forceinline__ void member_reduce(double (&v)[NV], double* partials, BMember* m, int tile,
                                              const Post& post) {
  block_sum<NV>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(size_t)tile * NV + q] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(&m->ticket, 1u);
    last = (t == (unsigned)m->ntiles - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int b = threadIdx.x; b < m->ntiles; b += blockDim.x)
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] += __ldcg(partials + (size_t)(m->tile0 + b) * NV + q);
  block_sum<NV>(acc);
  if (threadIdx.x == 0) {
    post(m, acc);
    m->ticket = 0u;
  }
}

// ------------------------------------------------------------------ posts

struct BPostOuter {
  int* active;
  __device__ void operator()(BMember* m, const double* v) const {
    const double rr = v[0];
    if (m->outer == 0) m->bb = rr;  // x = 0: r = b
    m->rr_outer = rr;
    m->outer += 1;
    m->e_valid = 0;
    int done = -1;
    if (!(rr == rr) || rr > 1.7e308) done = PDEB200_ERR_BREAKDOWN;
    else if (m->bb == 0.0 || rr <= m->tol2 * m->bb) done = PDEB200_OK;
    else if (m->outer > m->max_outer) done = PDEB200_ERR_NOT_CONVERGED;
    if (done >= 0) {
      m->status = done;
      m->state = kBDone;
      atomicSub(active, 1);
    } else {
      m->state = kBInnerStart;
      m->inner = 0;
      m->rr0 = rr;
      m->rr = rr;
      // the inner solve only has to take |r|^2 from rr to the target: on the
      // last refinement step that is less than inner_tol (a factor 4 of
      // margin on |r| for the FP32 operator's rounding)
      m->tol2_step = fmax(m->tol2_inner, fmin(0.01, 0.0625 * m->tol2 * m->bb / rr));
    }
  }
};

struct BPostPQ {
  __device__ void operator()(BMember* m, const double* v) const {
    const double pq = v[0];
    if (pq > 0.0 && pq < 1.7e308 && m->rz > 0.0) {
      m->alpha = m->rz / pq;
    } else {
      m->state = kBNeedOuter;  // breakdown: restart from the current refinement
    }
  }
};

struct BPostUpdate {
  __device__ void operator()(BMember* m, const double* v) const {
    const double rr = v[0];
    m->inner += 1;
    m->inner_total += 1;
    m->rr = rr;
    if (!(rr == rr) || rr > 1.7e308) {
      m->e_valid = 0;
      m->state = kBNeedOuter;
      return;
    }
    m->e_valid = 1;
    if (rr <= m->tol2_step * m->rr0 || m->inner >= m->max_inner) m->state = kBNeedOuter;
  }
};

struct BPostRZ {
  __device__ void operator()(BMember* m, const double* v) const {
    const double rz = v[0];
    if (!(rz > 0.0) || rz > 1.7e308) {
      m->state = kBNeedOuter;
      return;
    }
    if (m->state == kBInnerStart) {
      m->first = 1;
      m->beta = 0.0;
      m->state = kBInnerRun;
    } else {
      m->first = 0;
      m->beta = rz / m->rz;
    }
    m->rz = rz;
  }
};

// --------------------------------------------------------------- kernels

constexpr int kBThreads = 256;
// resident blocks per SM asked of the tile kernels (6: a 40-register cap):
// they are latency-bound, so more warps in flight beat more registers (the
// smoother takes 8, prolongation and the FP32 apply 5, restriction 4 to
// avoid spilling)
constexpr int kBMinBlocks = 6;

// Folded right-hand side b64 = -f - (face shift) and x64 = 0 on level 0.
__global__ void __launch_bounds__(kBThreads) kb_rhs(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                    const BMember* __restrict__ mem) {
  const BTile T = tiles[blockIdx.x];
  const BLevel& L = lv[T.lev];
  const BMember& m = mem[T.member];
  const double* k64 = m.k64;
  const double* f64 = m.f64;
  double* b64 = m.b64;
  double* x64 = m.x64;
  tile_columns(T, [&](int i, int j) {
    for (int kk = T.z0; kk < T.z1; ++kk) {
      const long long id = bid(L.g, i, j, kk);
      double sh = 0.0;
      (void)bstencil<double, double>(L, k64, i, j, kk, id, &sh);
      b64[id] = -(f64 ? f64[id] : 0.0) - sh;
      x64[id] = 0.0;
    }
  });
}

// x64 += e for members about to take an outer step with a pending correction.
__global__ void __launch_bounds__(kBThreads) kb_xupdate(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                        const BMember* mem) {
  const BTile T = tiles[blockIdx.x];
  const BMember* m = mem + T.member;
  if (bstate(m) != kBNeedOuter || !__ldcg(&m->e_valid)) return;
  const int nx = lv[T.lev].g.nx, ny = lv[T.lev].g.ny;
  double* __restrict__ x = m->x64;
  const float* __restrict__ e = m->e;
  tile_columns(T, [&](int i, int j) {
    for (int kk = T.z0; kk < T.z1; ++kk) {
      const long long id = ((long long)kk * ny + j) * nx + i;
      x[id] += double(e[id]);
    }
  });
}

// Outer FP64 residual r = b - A x; the FP32 copy is the inner right-hand side.
__global__ void __launch_bounds__(kBThreads) kb_outer(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                      BMember* mem, double* partials, int* active) {
  const BTile T = tiles[blockIdx.x];
  BMember* m = mem + T.member;
  if (bstate(m) != kBNeedOuter) return;
  const BLevel& L = lv[T.lev];
  const double* __restrict__ x = m->x64;
  const double* __restrict__ b = m->b64;
  float* __restrict__ r32 = L.b;
  const double* k64 = m->k64;
  const int nx = L.g.nx, dim = L.g.dim;
  const long long sxy = L.g.sxy;
  const bool is3 = dim == 3;
  double acc[1] = {0.0};
  tile_columns(T, [&](int i, int j) {
    long long id = bid(L.g, i, j, T.z0);
    double zm = is3 ? x[id - sxy] : 0.0;
    double zc = x[id];
    for (int kk = T.z0; kk < T.z1; ++kk, id += sxy) {
      const double zp = is3 ? x[id + sxy] : 0.0;
      const Stencil<double> s = bstencil<double, double>(L, k64, i, j, kk, id, nullptr);
      const double v = b[id] - (s.c * zc + nb_sum<double>(s, x[id + 1], x[id - 1], x[id + nx], x[id - nx], zp, zm,
                                                           dim));
      r32[id] = float(v);
      acc[0] += v * v;
      zm = zc;
      zc = zp;
    }
  });
  member_reduce<1>(acc, partials, m, blockIdx.x, BPostOuter{active});
}

// q = A p (FP32 operator, FP32 k), sum p.q in FP64.
__global__ void __launch_bounds__(kBThreads, 5) kb_apply_pq(const BTile* __restrict__ tiles,
                                                         const BLevel* __restrict__ lv, BMember* mem,
                                                         double* partials) {
  const BTile T = tiles[blockIdx.x];
  BMember* m = mem + T.member;
  if (bstate(m) != kBInnerRun) return;
  const BLevel& L = lv[T.lev];
  const float* __restrict__ p = m->p;
  float* __restrict__ q = m->q;
  FStencil<float> S;
  S.load(L, m->k32);
  const int nx = S.nx, sxy = S.sxy;
  double acc[1] = {0.0};
  // one branch on the tile's dimension; inside, D is a constant
  auto columns = [&](auto dc) {
    constexpr int D = decltype(dc)::value;
    tile_columns(T, [&](int i, int j) {
      int id = (T.z0 * S.ny + j) * nx + i;
      float zm = D == 3 ? p[id - sxy] : 0.f;
      float zc = p[id];
      for (int kk = T.z0; kk < T.z1; ++kk, id += sxy) {
        const float zp = D == 3 ? p[id + sxy] : 0.f;
        const Stencil<float> s = S.template at<D>(i, j, kk, id);
        const float v = s.c * zc + nb_sum<float>(s, p[id + 1], p[id - 1], p[id + nx], p[id - nx], zp, zm, D);
        q[id] = v;
        acc[0] += double(zc) * double(v);
        zm = zc;
        zc = zp;
      }
    });
  };
  if (S.dim == 3)
    columns(std::integral_constant<int, 3>{});
  else
    columns(std::integral_constant<int, 2>{});
  member_reduce<1>(acc, partials, m, blockIdx.x, BPostPQ{});
}

// e (+)= alpha p, r -= alpha q, sum r.r in FP64.
__global__ void __launch_bounds__(kBThreads) kb_update(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                       BMember* mem, double* partials) {
  const BTile T = tiles[blockIdx.x];
  BMember* m = mem + T.member;
  if (bstate(m) != kBInnerRun) return;
  const int nx = lv[T.lev].g.nx, ny = lv[T.lev].g.ny;
  float* __restrict__ r = lv[T.lev].b;
  const float* __restrict__ p = m->p;
  const float* __restrict__ q = m->q;
  float* __restrict__ e = m->e;
  const float a = float(__ldcg(&m->alpha));
  const bool first = __ldcg(&m->inner) == 0;
  double acc[1] = {0.0};
  tile_columns(T, [&](int i, int j) {
    for (int kk = T.z0; kk < T.z1; ++kk) {
      const long long id = ((long long)kk * ny + j) * nx + i;
      e[id] = first ? a * p[id] : e[id] + a * p[id];
      const float rv = r[id] - a * q[id];
      r[id] = rv;
      acc[0] += double(rv) * double(rv);
    }
  });
  member_reduce<1>(acc, partials, m, blockIdx.x, BPostUpdate{});
}

// sum r.z in FP64 (starts a new inner solve or gives beta).
__global__ void __launch_bounds__(kBThreads) kb_rz(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                   BMember* mem, double* partials) {
  const BTile T = tiles[blockIdx.x];
  BMember* m = mem + T.member;
  if (!vcycle_state(bstate(m))) return;
  const int nx = lv[T.lev].g.nx, ny = lv[T.lev].g.ny;
  const float* __restrict__ r = lv[T.lev].b;
  const float* __restrict__ z = lv[T.lev].x;
  double acc[1] = {0.0};
  tile_columns(T, [&](int i, int j) {
    for (int kk = T.z0; kk < T.z1; ++kk) {
      const long long id = ((long long)kk * ny + j) * nx + i;
      acc[0] += double(r[id]) * double(z[id]);
    }
  });
  member_reduce<1>(acc, partials, m, blockIdx.x, BPostRZ{});
}

// p = z + beta p (p = z when the inner solve starts).
__global__ void __launch_bounds__(kBThreads) kb_pupdate(const BTile* __restrict__ tiles,
                                                        const BLevel* __restrict__ lv, const BMember* mem) {
  const BTile T = tiles[blockIdx.x];
  const BMember* m = mem + T.member;
  if (bstate(m) != kBInnerRun) return;
  const int nx = lv[T.lev].g.nx, ny = lv[T.lev].g.ny;
  const float* __restrict__ z = lv[T.lev].x;
  float* __restrict__ p = m->p;
  const bool first = __ldcg(&m->first) != 0;
  const float bt = float(__ldcg(&m->beta));
  tile_columns(T, [&](int i, int j) {
    for (int kk = T.z0; kk < T.z1; ++kk) {
      const long long id = ((long long)kk * ny + j) * nx + i;
      p[id] = first ? z[id] : z[id] + bt * p[id];
    }
  });
}

// One red-black colour pass of the V-cycle smoother on level tiles. from_zero:
// x is taken as zero (first pass of a level): the colour's nodes get b/diag,
// the other colour's nodes 0.
template <typename KT>
__global__ void __launch_bounds__(kBThreads, 8) kb_smooth(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                       const BMember* mem, int color, int from_zero) {
  const BTile T = tiles[blockIdx.x];
  if (T.coarse) return;
  if (!vcycle_state(bstate(mem + T.member))) return;
  const BLevel& L = lv[T.lev];
  float* __restrict__ x = L.x;
  // In one colour pass no node is both written and read (updated nodes read
  // only the other colour), so the reads go through a separate read-only
  // view and the loads of later nodes can overlap earlier stores.
  const float* __restrict__ xr = L.x;
  const float* __restrict__ b = L.b;
  FStencil<KT> S;
  S.load(L, static_cast<const KT*>(L.kh));
  const int nx = S.nx, sxy = S.sxy, dim = S.dim;
  const bool is3 = dim == 3;
  if (!is3 && !from_zero) {
    // 2D: threads walk only the cells of the colour being updated
    const int half = (int(T.w) + 1) >> 1;
    const int total = int(T.h) * half;
    const int i0 = 1 + T.x0;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int row = t / half, c = t - row * half;
      const int j = 1 + T.y0 + row;
      const int ra = 2 * c + ((i0 + j + color) & 1);
      if (ra >= int(T.w)) continue;
      const int i = i0 + ra;
      const int id = j * nx + i;
      const Stencil<float> s = S.template at<2>(i, j, 0, id);
      x[id] = (b[id] - nb_sum<float>(s, xr[id + 1], xr[id - 1], xr[id + nx], xr[id - nx], 0.f, 0.f, 2)) / s.c;
    }
    return;
  }
  tile_columns(T, [&](int i, int j) {
    if (from_zero) {
      for (int kk = T.z0; kk < T.z1; ++kk) {
        const int id = (kk * S.ny + j) * nx + i;
        if (((i + j + kk) & 1) == color) {
          const Stencil<float> s = S.at(i, j, kk, id);
          x[id] = b[id] / s.c;
        } else {
          x[id] = 0.f;
        }
      }
    } else {
      // 3D here (the 2D pass returned above): the z loads are not predicated
#pragma unroll 2
      for (int kk = T.z0 + ((i + j + T.z0 + color) & 1); kk < T.z1; kk += 2) {
        const int id = (kk * S.ny + j) * nx + i;
        const Stencil<float> s = S.template at<3>(i, j, kk, id);
        const float zp = xr[id + sxy];
        const float zm = xr[id - sxy];
        x[id] = (b[id] - nb_sum<float>(s, xr[id + 1], xr[id - 1], xr[id + nx], xr[id - nx], zp, zm, 3)) / s.c;
      }
    }
  });
}

// Level residual r = b - A x on level tiles.
template <typename KT>
__global__ void __launch_bounds__(kBThreads, kBMinBlocks) kb_residual(const BTile* __restrict__ tiles,
                                                         const BLevel* __restrict__ lv, const BMember* mem) {
  const BTile T = tiles[blockIdx.x];
  if (T.coarse) return;
  if (!vcycle_state(bstate(mem + T.member))) return;
  const BLevel& L = lv[T.lev];
  const float* __restrict__ x = L.x;
  const float* __restrict__ b = L.b;
  float* __restrict__ r = L.r;
  FStencil<KT> S;
  S.load(L, static_cast<const KT*>(L.kh));
  const int nx = S.nx, sxy = S.sxy;
  // one branch on the tile's dimension; inside, D is a constant
  auto columns = [&](auto dc) {
    constexpr int D = decltype(dc)::value;
    tile_columns(T, [&](int i, int j) {
      int id = (T.z0 * S.ny + j) * nx + i;
      float zm = D == 3 ? x[id - sxy] : 0.f;
      float zc = x[id];
      for (int kk = T.z0; kk < T.z1; ++kk, id += sxy) {
        const float zp = D == 3 ? x[id + sxy] : 0.f;
        const Stencil<float> s = S.template at<D>(i, j, kk, id);
        r[id] = b[id] - (s.c * zc + nb_sum<float>(s, x[id + 1], x[id - 1], x[id + nx], x[id - nx], zp, zm, D));
        zm = zc;
        zc = zp;
      }
    });
  };
  if (S.dim == 3)
    columns(std::integral_constant<int, 3>{});
  else
    columns(std::integral_constant<int, 2>{});
}

// Coarsest-level solve inside one block: `sweeps` red-black sweeps from zero
// in FP64 (shared memory when the grid has at most kBCoarseSmem nodes, else
// in place on the FP32 field with FP64 arithmetic).
constexpr int kBCoarseSmem = 256;

template <typename KT>
__device__ __noinline__ void bcoarse_solve(const BLevel& C, int sweeps) {
  __shared__ double cs[kBCoarseSmem];
  const KT* k = static_cast<const KT*>(C.kh);
  const GridDev& g = C.g;
  const int kb = g.dim == 3 ? 1 : 0, ke = g.dim == 3 ? g.nz - 1 : 1;
  const int ni = g.nx - 2, nj = g.ny - 2, nk = ke - kb;
  const int total = ni * nj * nk;
  const bool smem = g.n <= kBCoarseSmem;
  float* x = C.x;
  const float* b = C.b;
  if (smem) {
    for (int t = threadIdx.x; t < (int)g.n; t += blockDim.x) cs[t] = 0.0;
  } else {
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int i = 1 + t % ni, j = 1 + (t / ni) % nj, kk = kb + t / (ni * nj);
      x[bid(g, i, j, kk)] = 0.f;
    }
  }
  __syncthreads();
  if (total == 1 && sweeps > 1) sweeps = 1;  // one interior node: the first sweep is the fixed point
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int i = 1 + t % ni, j = 1 + (t / ni) % nj, kk = kb + t / (ni * nj);
        if (((i + j + kk) & 1) != color) continue;
        const long long id = bid(g, i, j, kk);
        const Stencil<double> st = bstencil<double, KT>(C, k, i, j, kk, id, nullptr);
        double v;
        if (smem) {
          const int q = (int)id, nx = g.nx, sxy = (int)g.sxy;
          v = st.xp * cs[q + 1] + st.xm * cs[q - 1] + st.yp * cs[q + nx] + st.ym * cs[q - nx];
          if (g.dim == 3) v += st.zp * cs[q + sxy] + st.zm * cs[q - sxy];
          cs[q] = (double(b[id]) - v) / st.c;
        } else {
          v = st.xp * double(x[id + 1]) + st.xm * double(x[id - 1]) + st.yp * double(x[id + g.nx]) +
              st.ym * double(x[id - g.nx]);
          if (g.dim == 3) v += st.zp * double(x[id + g.sxy]) + st.zm * double(x[id - g.sxy]);
          x[id] = float((double(b[id]) - v) / st.c);
        }
      }
      __syncthreads();
    }
  if (smem)
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      const int i = 1 + t % ni, j = 1 + (t / ni) % nj, kk = kb + t / (ni * nj);
      const long long id = bid(g, i, j, kk);
      x[id] = float(cs[id]);
    }
}

// Restriction into level-(l+1) tiles: coarse b = Ext^T P^T r_fine at interior
// coarse nodes (the boundary-closure fold recomputes the full weight of each
// Neumann/Robin boundary node that feeds an interior one). A whole-grid tile
// of a coarsest level then solves that level in the same block.
// Boundary-closure fold of the restriction at an interior coarse node next to
// a face: coef x full weight of each boundary node whose chain ends there.
__device__ __noinline__ double brestrict_fold(const GridDev& gf, const GridDev& gc, const float* __restrict__ rf,
                                              int I, int J, int K, int dxl, int dxh, int dyl, int dyh, int dzl,
                                              int dzh) {
  double fold = 0.0;
  for (int dk = dzl; dk <= dzh; ++dk)
    for (int dj = dyl; dj <= dyh; ++dj)
      for (int di = dxl; di <= dxh; ++di) {
        if (di == 0 && dj == 0 && dk == 0) continue;
        int ci = I + di, cj = J + dj, ck = K + dk;
        const double coef = ext_chain(gc, ci, cj, ck);
        if (coef != 0.0 && ci == I && cj == J && ck == K)
          fold += coef * full_weight<float>(gf, gc, rf, I + di, J + dj, K + dk);
      }
  return fold;
}

// One coarse column of the restriction in the general form (any transfer
// map), out of line so the common nested path keeps few registers.
__device__ __noinline__ void brestrict_column_general(const BLevel& F, const BLevel& C, const float* __restrict__ rf,
                                                      float* __restrict__ bc, const BTile& T, int I, int J, int dxl,
                                                      int dxh, int dyl, int dyh, bool zmarch, bool zsame) {
  const GridDev& gc = C.g;
  FwColumn<float> col;
  col.init(F.g, gc, rf, I, J);
  // nested z: fine plane 2K+1 feeds coarse planes K and K+1 (sum kept)
  double below = zmarch && gc.dim == 3 && !zsame ? col.plane(2 * T.z0 - 1) : 0.0;
  for (int K = T.z0; K < T.z1; ++K) {
    double acc;
    if (!zmarch) {
      acc = full_weight<float>(F.g, gc, rf, I, J, K);
    } else if (gc.dim != 3) {
      acc = col.plane(0);
    } else if (zsame) {
      acc = col.plane(K);
    } else {
      const double mid = col.plane(2 * K);
      const double above = 2 * K + 1 <= F.g.nz - 1 ? col.plane(2 * K + 1) : 0.0;
      acc = 0.25 * below + 0.5 * mid + 0.25 * above;
      below = above;
    }
    const int dzl = gc.dim == 3 && K == 1 ? -1 : 0, dzh = gc.dim == 3 && K == gc.nz - 2 ? 1 : 0;
    if (dxl | dxh | dyl | dyh | dzl | dzh) {
      for (int dk = dzl; dk <= dzh; ++dk)
        for (int dj = dyl; dj <= dyh; ++dj)
          for (int di = dxl; di <= dxh; ++di) {
            if (di == 0 && dj == 0 && dk == 0) continue;
            int ci = I + di, cj = J + dj, ck = K + dk;
            const double coef = ext_chain(gc, ci, cj, ck);
            if (coef != 0.0 && ci == I && cj == J && ck == K)
              acc += coef * full_weight<float>(F.g, gc, rf, I + di, J + dj, K + dk);
          }
    }
    bc[bid(gc, I, J, K)] = float(acc);
  }
}

template <typename KT>
__global__ void __launch_bounds__(kBThreads, 4) kb_restrict(const BTile* __restrict__ tiles,
                                                         const BLevel* __restrict__ lv, const BMember* mem,
                                                         int coarse_sweeps) {
  const BTile T = tiles[blockIdx.x];
  if (!vcycle_state(bstate(mem + T.member))) return;
  const BLevel& C = lv[T.lev];
  const BLevel& F = lv[C.prev];
  const GridDev& gc = C.g;
  const float* __restrict__ rf = F.r;
  float* __restrict__ bc = C.b;
  const bool zmarch = gc.dim != 3 || map_mode(F.g.nz, gc.nz) <= 1;
  const bool zsame = gc.dim == 3 && gc.nz == F.g.nz;
  const int xm = map_mode(F.g.nx, gc.nx), ym = map_mode(F.g.ny, gc.ny);
  // nested 2:1 or identity in every dimension: FP32 weights {1/4, 1/2, 1/4}
  // (or {0, 1, 0}) on the three fine nodes around each interior coarse node,
  // always inside the fine grid, no clipping
  const bool fast = xm <= 1 && ym <= 1 && zmarch;
  const int fnx = F.g.nx;
  const long long fsxy = F.g.sxy;
  tile_columns(T, [&](int I, int J) {
    if (fast) {
      const int fi = (xm == 1 ? 2 * I : I) - 1, fj = (ym == 1 ? 2 * J : J) - 1;
      const float wx0 = xm == 1 ? 0.25f : 0.f, wx1 = xm == 1 ? 0.5f : 1.f;
      const float wy0 = ym == 1 ? 0.25f : 0.f, wy1 = ym == 1 ? 0.5f : 1.f;
      auto plane = [&](int fk) -> float {
        const float* r0 = rf + (long long)fk * fsxy + (long long)fj * fnx + fi;
        const float s0 = wx0 * r0[0] + wx1 * r0[1] + wx0 * r0[2];
        const float* r1 = r0 + fnx;
        const float s1 = wx0 * r1[0] + wx1 * r1[1] + wx0 * r1[2];
        const float* r2 = r1 + fnx;
        const float s2 = wx0 * r2[0] + wx1 * r2[1] + wx0 * r2[2];
        return wy0 * s0 + wy1 * s1 + wy0 * s2;
      };
      const int dxl = I == 1 ? -1 : 0, dxh = I == gc.nx - 2 ? 1 : 0;
      const int dyl = J == 1 ? -1 : 0, dyh = J == gc.ny - 2 ? 1 : 0;
      float below = gc.dim == 3 && !zsame ? plane(2 * T.z0 - 1) : 0.f;
      for (int K = T.z0; K < T.z1; ++K) {
        float acc;
        if (gc.dim != 3) {
          acc = plane(0);
        } else if (zsame) {
          acc = plane(K);
        } else {
          const float mid = plane(2 * K), above = plane(2 * K + 1);
          acc = 0.25f * below + 0.5f * mid + 0.25f * above;
          below = above;
        }
        const int dzl = gc.dim == 3 && K == 1 ? -1 : 0, dzh = gc.dim == 3 && K == gc.nz - 2 ? 1 : 0;
        if (dxl | dxh | dyl | dyh | dzl | dzh)
          acc = float(double(acc) + brestrict_fold(F.g, gc, rf, I, J, K, dxl, dxh, dyl, dyh, dzl, dzh));
        bc[bid(gc, I, J, K)] = acc;
      }
      return;
    }
    const int dxl = I == 1 ? -1 : 0, dxh = I == gc.nx - 2 ? 1 : 0;
    const int dyl = J == 1 ? -1 : 0, dyh = J == gc.ny - 2 ? 1 : 0;
    brestrict_column_general(F, C, rf, bc, T, I, J, dxl, dxh, dyl, dyh, zmarch, zsame);
  });
  if (T.coarse) {
    __syncthreads();
    bcoarse_solve<KT>(C, coarse_sweeps);
  }
}

// x_l += P Ext(x_{l+1}) on level-l tiles of members with a coarser level.
__global__ void __launch_bounds__(kBThreads, 5) kb_prolong(const BTile* __restrict__ tiles, const BLevel* __restrict__ lv,
                                                        const BMember* mem) {
  const BTile T = tiles[blockIdx.x];
  if (T.coarse) return;
  if (!vcycle_state(bstate(mem + T.member))) return;
  const BLevel& F = lv[T.lev];
  const BLevel& C = lv[F.next];
  const GridDev& gf = F.g;
  const GridDev& gc = C.g;
  const float* __restrict__ xc = C.x;
  float* __restrict__ xf = F.x;
  const int xmode = map_mode(gf.nx, gc.nx), ymode = map_mode(gf.ny, gc.ny);
  const int zmode = gf.dim == 3 ? map_mode(gf.nz, gc.nz) : 0;
  if (xmode <= 1 && ymode <= 1 && zmode <= 1) {
    // nested 2:1 or identity in every dimension: interpolation weights are 1
    // or 1/2, in FP32, loading only the coarse values a node uses
    tile_columns(T, [&](int i, int j) {
      const bool ax = xmode == 1 && (i & 1), ay = ymode == 1 && (j & 1);
      const int I0 = xmode == 1 ? i >> 1 : i, J0 = ymode == 1 ? j >> 1 : j;
      const int I1 = ax ? I0 + 1 : I0, J1 = ay ? J0 + 1 : J0;
      const bool xy_edge = I0 == 0 || I1 == gc.nx - 1 || J0 == 0 || J1 == gc.ny - 1;
      auto bil = [&](int K) -> float {
        const bool edge = xy_edge || (gf.dim == 3 && (K == 0 || K == gc.nz - 1));
        auto cv = [&](int I, int J) -> float {
          return edge ? float(ext_value(gc, xc, I, J, K)) : xc[(long long)K * gc.sxy + (long long)J * gc.nx + I];
        };
        const float c00 = cv(I0, J0);
        if (!ax && !ay) return c00;
        if (!ay) return 0.5f * (c00 + cv(I1, J0));
        if (!ax) return 0.5f * (c00 + cv(I0, J1));
        return 0.25f * ((c00 + cv(I1, J0)) + (cv(I0, J1) + cv(I1, J1)));
      };
      if (gf.dim != 3) {
        const long long id = bid(gf, i, j, 0);
        xf[id] += bil(0);
        return;
      }
      // march in z: each coarse plane's value is computed once and shared by
      // the fine planes it feeds
      int ka = -1, kb = -1;
      float va = 0.f, vb = 0.f;
      auto at = [&](int K) -> float {
        if (K == kb) return vb;
        if (K == ka) return va;
        ka = kb;
        va = vb;
        kb = K;
        vb = bil(K);
        return vb;
      };
      for (int k = T.z0; k < T.z1; ++k) {
        const int K0 = zmode == 1 ? k >> 1 : k;
        const bool az = zmode == 1 && (k & 1);
        const float v = az ? 0.5f * (at(K0) + at(K0 + 1)) : at(K0);
        const long long id = bid(gf, i, j, k);
        xf[id] += v;
      }
    });
    return;
  }
  tile_columns(T, [&](int i, int j) {
    int I0, J0;
    double tx, ty;
    coarse_pos(i, gf.nx, gc.nx, xmode, I0, tx);
    coarse_pos(j, gf.ny, gc.ny, ymode, J0, ty);
    const int I1 = tx != 0.0 ? I0 + 1 : I0, J1 = ty != 0.0 ? J0 + 1 : J0;
    const bool xy_edge = I0 == 0 || I1 == gc.nx - 1 || J0 == 0 || J1 == gc.ny - 1;
    // bilinear x-y value on coarse plane K, kept for the fine planes it feeds
    auto bilinear = [&](int K) -> double {
      double c00, c10, c01, c11;
      if (!xy_edge && !(gf.dim == 3 && (K == 0 || K == gc.nz - 1))) {
        const long long a = (long long)K * gc.sxy;
        const long long r0 = (long long)J0 * gc.nx, r1 = (long long)J1 * gc.nx;
        c00 = double(xc[a + r0 + I0]);
        c10 = double(xc[a + r0 + I1]);
        c01 = double(xc[a + r1 + I0]);
        c11 = double(xc[a + r1 + I1]);
      } else {
        c00 = ext_value(gc, xc, I0, J0, K);
        c10 = ext_value(gc, xc, I1, J0, K);
        c01 = ext_value(gc, xc, I0, J1, K);
        c11 = ext_value(gc, xc, I1, J1, K);
      }
      const double x0 = (1.0 - tx) * c00 + tx * c10, x1 = (1.0 - tx) * c01 + tx * c11;
      return (1.0 - ty) * x0 + ty * x1;
    };
    int ka = -1, kb = -1;
    double va = 0.0, vb = 0.0;
    auto at = [&](int K) -> double {
      if (K == ka) return va;
      if (K == kb) return vb;
      const double v = bilinear(K);
      ka = kb;
      va = vb;
      kb = K;
      vb = v;
      return v;
    };
    for (int k = T.z0; k < T.z1; ++k) {
      int K0 = 0;
      double tz = 0.0;
      if (gf.dim == 3) coarse_pos(k, gf.nz, gc.nz, zmode, K0, tz);
      const double y0 = at(K0);
      const double y1 = tz != 0.0 ? at(K0 + 1) : y0;
      const double v = (1.0 - tz) * y0 + tz * y1;
      const long long id = bid(gf, i, j, k);
      xf[id] = float(double(xf[id]) + v);
    }
  });
}

// Boundary nodes of each member's FP64 solution from the closures (reference
// phase order, Dirichlet last); one block per member.
__global__ void __launch_bounds__(kBThreads) kb_fill_boundary(const BLevel* __restrict__ lv,
                                                              const BMember* __restrict__ mem) {
  const BMember* m = mem + blockIdx.x;
  const GridDev& g = lv[m->level0].g;
  double* u = m->x64;
  const long long nyz = (long long)g.ny * g.nz, nxz = (long long)g.nx * g.nz, nxy = (long long)g.nx * g.ny;
  const long long total = 2 * nyz + 2 * nxz + (g.dim == 3 ? 2 * nxy : 0);
  // one thread per face node; a node shared by faces is written by the first
  // face (in face order) that contains it
  for (long long t = threadIdx.x; t < total; t += blockDim.x) {
    int i, j, k, f;
    long long q = t;
    if (q < 2 * nyz) {
      f = q < nyz ? kLeft : kRight;
      i = q < nyz ? 0 : g.nx - 1;
      q %= nyz;
      j = int(q % g.ny);
      k = int(q / g.ny);
    } else if ((q -= 2 * nyz) < 2 * nxz) {
      f = q < nxz ? kBottom : kTop;
      j = q < nxz ? 0 : g.ny - 1;
      q %= nxz;
      i = int(q % g.nx);
      k = int(q / g.nx);
    } else {
      q -= 2 * nxz;
      f = q < nxy ? kFront : kBack;
      k = q < nxy ? 0 : g.nz - 1;
      q %= nxy;
      i = int(q % g.nx);
      j = int(q / g.nx);
    }
    const bool on[6] = {i == 0, i == g.nx - 1, j == 0, j == g.ny - 1, g.dim == 3 && k == 0,
                        g.dim == 3 && k == g.nz - 1};
    int owner = -1;
    for (int w = 0; w < 6 && owner < 0; ++w)
      if (on[w]) owner = w;
    if (owner != f) continue;
    u[bid(g, i, j, k)] = boundary_final(g, u, i, j, k, true);
  }
}

}  // namespace pdeb
