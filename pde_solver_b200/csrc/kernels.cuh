// Kernels of libpdeb200. All stencil kernels use the same mapping: a thread
// owns an (i,j) column and marches over a chunk of k, keeping the three
// z-planes of the field it reads in registers (x/y neighbours come through
// L1/L2). Blocks are 32 x 8 threads: a warp reads 32 consecutive doubles of
// a row (fully coalesced 256 B).
//
// Every kernel of an iterative solve takes `ctl`, a device control block: when
// ctl->done is set (convergence or breakdown found on the device) the kernel
// returns at once. The host can therefore enqueue several iterations ahead and
// poll lazily while the result stays exactly the one of stopping at the first
// converged iteration.
#pragma once

#include "device.cuh"

namespace pdeb {

constexpr int kBx = 32;
constexpr int kBy = 8;
// capacity (in blocks) of the reduction partial buffers; launch shapes stay below it
constexpr long long kMaxGridBlocks = 1LL << 17;

struct Ctl {
  int done;        // every kernel of the solve returns at once
  int stop;        // relaxation: no further sweeps; closures still run
  int status;      // pdeb200_status recorded with done/stop
  int iter;        // completed iterations
  int max_iter;
  int pad;
  double tol;      // absolute threshold (reference rules)
  double tol2;     // squared threshold on the monitored norm (relative rule)
  double brk;      // breakdown threshold on Krylov denominators
  double rr;       // last monitored squared norm
  double rz, pq, alpha, beta;             // CG family
  double rho, rho_prev, omega, tt, ts;    // BiCGStab family
  double bb;       // |b|^2
  double delta;    // relaxation max |du|
  double aux[8];
};

__device__ __forceinline__ bool ctl_skip(const Ctl* c) { return c && *((volatile const int*)&c->done); }

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization (launch_dep on the host) may be scheduled while the previous
// kernel of the stream is still running. grid_dep_wait() returns once that
// kernel has completed and its writes are visible (at once for an ordinary
// launch); grid_dep_release() lets the next such launch be scheduled. The
// kernels launch_dep launches call both through ctl_skip_dep, before their
// first memory access, so at most one kernel is scheduled ahead and it
// touches no memory until its predecessor is done: the results are those of
// plain stream order.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ bool ctl_skip_dep(const Ctl* c) {
  grid_dep_wait();
  grid_dep_release();
  return ctl_skip(c);
}
__device__ __forceinline__ bool ctl_stopped(const Ctl* c) {
  return c && (*((volatile const int*)&c->done) || *((volatile const int*)&c->stop));
}

__device__ __forceinline__ void column_range(const GridDev& g, int& k0, int& k1) {
  // interior z range split into gridDim.z chunks
  const int kb = g.dim == 3 ? 1 : 0;
  const int ke = g.dim == 3 ? g.nz - 1 : 1;
  const int len = ke - kb;
  const int chunk = (len + gridDim.z - 1) / gridDim.z;
  k0 = kb + blockIdx.z * chunk;
  k1 = min(ke, k0 + chunk);
}

// ------------------------------------------------------------ folded apply

// Planes ahead of the current trip that the apply and the residual prefetch
// into L2 (x, k and b of two planes per trip): at 257^3 the apply goes from
// 141 to 116 us and the residual from 141 to 127 us; 2, 6 and 8 planes ahead
// are slower. The colour pass is slower with any prefetch distance.
constexpr int kPfPlanes = 4;

// The columns of one thread of k_apply_folded / k_residual_folded (RES: r = b
// - A x, else y = A x). D is the grid dimension: the kernels branch on it
// once, and the stencil helpers take it as a constant (with the prefetch,
// 257^3 apply 116 -> 105 us, residual 127 -> 121 us). acc sums x*y (apply) or
// r*r (residual) when NV > 0.
template <int D, bool RES, int NV, class Coef, typename T, typename TB>
__device__ __forceinline__ void stencil_columns(const GridDev& g, const Coef& cf, const T* __restrict__ x,
                                                const TB* __restrict__ b, T* __restrict__ y, double& acc) {
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(g, k0, k1);
  if (!(i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) || k0 >= k1) return;
  long long id = ((long long)k0 * g.ny + j) * g.nx + i;
  T zm = D == 3 ? x[id - g.sxy] : T(0);
  T zc = x[id];
  int k = k0;
  // two planes per trip, all loads before the stores (with one plane per
  // trip the kernels are latency-bound)
  for (; k + 1 < k1; k += 2, id += 2 * g.sxy) {
    if (k + kPfPlanes + 1 < g.nz) {
      const long long a = id + kPfPlanes * g.sxy;
      pf_l2(x + a);
      pf_l2(x + a + g.sxy);
      cf.prefetch(a);
      cf.prefetch(a + g.sxy);
      if constexpr (RES) {
        pf_l2(b + a);
        pf_l2(b + a + g.sxy);
      }
    }
    const long long id2 = id + g.sxy;
    const T z1 = x[id2];
    const T z2 = x[id2 + g.sxy];
    const T xp1 = x[id + 1], xm1 = x[id - 1], yp1 = x[id + g.nx], ym1 = x[id - g.nx];
    const T xp2 = x[id2 + 1], xm2 = x[id2 - 1], yp2 = x[id2 + g.nx], ym2 = x[id2 - g.nx];
    T b1 = T(0), b2 = T(0);
    if constexpr (RES) {
      b1 = T(b[id]);
      b2 = T(b[id2]);
    }
    Stencil<T> s = cf.template at<T, D>(g, id);
    Stencil<T> s2 = cf.template at<T, D>(g, id2);
    fold_faces<T, D>(g, i, j, k, s, nullptr);
    fold_faces<T, D>(g, i, j, k + 1, s2, nullptr);
    const T a1 = s.c * zc + nb_sum<T>(s, xp1, xm1, yp1, ym1, z1, zm, D);
    const T a2 = s2.c * z1 + nb_sum<T>(s2, xp2, xm2, yp2, ym2, z2, zc, D);
    const T v = RES ? b1 - a1 : a1;
    const T v2 = RES ? b2 - a2 : a2;
    y[id] = v;
    y[id2] = v2;
    if constexpr (NV > 0) {
      acc += RES ? double(v) * double(v) : double(zc) * double(v);
      acc += RES ? double(v2) * double(v2) : double(z1) * double(v2);
    }
    zm = z1;
    zc = z2;
  }
  for (; k < k1; ++k, id += g.sxy) {
    const T zp = D == 3 ? x[id + g.sxy] : T(0);
    Stencil<T> s = cf.template at<T, D>(g, id);
    fold_faces<T, D>(g, i, j, k, s, nullptr);
    const T a = s.c * zc + nb_sum<T>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, D);
    const T v = RES ? T(b[id]) - a : a;
    y[id] = v;
    if constexpr (NV > 0) acc += RES ? double(v) * double(v) : double(zc) * double(v);
    zm = zc;
    zc = zp;
  }
}

// y = A_fold x on interior nodes (boundary rows of y untouched), with optional
// fused sum(w * y) (w = x for p.Ap).
template <class Coef, typename T, int NV, class Post>
__global__ void __launch_bounds__(kBx* kBy) k_apply_folded(GridDev g, Coef cf, const T* __restrict__ x,
                                                           T* __restrict__ y, RedSlot slot, Post post,
                                                           const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  double acc[(NV > 0 ? NV : 1)] = {0.0};
  if (g.dim == 3)
    stencil_columns<3, false, NV, Coef, T, T>(g, cf, x, nullptr, y, acc[0]);
  else
    stencil_columns<2, false, NV, Coef, T, T>(g, cf, x, nullptr, y, acc[0]);
  if constexpr (NV > 0) grid_reduce<(NV > 0 ? NV : 1), false>(acc, slot, post);
}

// r = b - A_fold x on interior nodes, optional fused |r|^2. Capped at 64
// registers (4 blocks/SM, some spill): at 257^3 121 us, against 124 us with
// 3 blocks/SM.
template <class Coef, typename T, typename TB, int NV, class Post>
__global__ void __launch_bounds__(kBx* kBy, 4) k_residual_folded(GridDev g, Coef cf, const T* __restrict__ x,
                                                              const TB* __restrict__ b, T* __restrict__ r,
                                                              RedSlot slot, Post post, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  double acc[(NV > 0 ? NV : 1)] = {0.0};
  if (g.dim == 3)
    stencil_columns<3, true, NV, Coef, T, TB>(g, cf, x, b, r, acc[0]);
  else
    stencil_columns<2, true, NV, Coef, T, TB>(g, cf, x, b, r, acc[0]);
  if constexpr (NV > 0) grid_reduce<(NV > 0 ? NV : 1), false>(acc, slot, post);
}

// Folded right-hand side b = -f - sum_faces w*c0 (boundary entries 0).
template <class Coef>
__global__ void __launch_bounds__(kBx* kBy) k_folded_rhs(GridDev g, Coef cf, const double* __restrict__ f,
                                                         double f_const, double* __restrict__ b) {
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(g, k0, k1);
  if (!(i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2)) return;
  for (int k = k0; k < k1; ++k) {
    const long long id = ((long long)k * g.ny + j) * g.nx + i;
    Stencil<double> s = cf.template at<double>(g, id);
    double sh = 0.0;
    fold_faces<double>(g, i, j, k, s, &sh);
    b[id] = -(f ? f[id] : f_const) - sh;
  }
}

// The columns of one thread of a colour pass. D is the grid dimension: the
// kernel branches on it once, so the field loads of the 3D form are not
// predicated and are all issued before the stores (with run-time dimension
// tests on them the 257^3 pass takes 120 instead of 107 us). HD is the
// dimension handed to the stencil helpers (0: their run-time test); the 3D
// form keeps the run-time test there, which measured faster than the
// constant (118 us).
template <int D, int HD, class Coef, typename T, typename TB, bool ZERO, bool DOT>
__device__ __forceinline__ void rbgs_columns(const GridDev& g, const Coef& cf, const TB* __restrict__ b,
                                             T* __restrict__ x, int color, double& acc) {
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(g, k0, k1);
  if (!(i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) || k0 >= k1) return;
  const int nd = HD ? HD : g.dim;
  int k = k0 + ((i + j + k0 + color) & 1);
  auto ld = [&](long long q) -> T {
    if constexpr (ZERO) return T(0);
    return x[q];
  };
  // nodes k and k+2 of one colour per trip: neither reads the other (their
  // neighbours are all of the other colour), so both nodes' loads are issued
  // before either store
  for (; k + 2 < k1; k += 4) {
    const long long id = ((long long)k * g.ny + j) * g.nx + i, id2 = id + 2 * g.sxy;
    Stencil<T> s = cf.template at<T, HD>(g, id);
    Stencil<T> s2 = cf.template at<T, HD>(g, id2);
    const T b1 = T(b[id]), b2 = T(b[id2]);
    const T zm = D == 3 ? ld(id - g.sxy) : T(0);
    const T mid = D == 3 ? ld(id + g.sxy) : T(0);  // zp of node k, zm of node k+2
    const T zp2 = D == 3 ? ld(id2 + g.sxy) : T(0);
    const T xp1 = ld(id + 1), xm1 = ld(id - 1), yp1 = ld(id + g.nx), ym1 = ld(id - g.nx);
    const T xp2 = ld(id2 + 1), xm2 = ld(id2 - 1), yp2 = ld(id2 + g.nx), ym2 = ld(id2 - g.nx);
    fold_faces<T, HD>(g, i, j, k, s, nullptr);
    fold_faces<T, HD>(g, i, j, k + 2, s2, nullptr);
    const T v1 = (b1 - nb_sum<T>(s, xp1, xm1, yp1, ym1, mid, zm, nd)) / s.c;
    const T v2 = (b2 - nb_sum<T>(s2, xp2, xm2, yp2, ym2, zp2, mid, nd)) / s2.c;
    x[id] = v1;
    x[id2] = v2;
    if constexpr (DOT) {
      acc += double(b1) * double(v1);
      acc += double(b2) * double(v2);
    }
  }
  for (; k < k1; k += 2) {
    const long long id = ((long long)k * g.ny + j) * g.nx + i;
    Stencil<T> s = cf.template at<T, HD>(g, id);
    fold_faces<T, HD>(g, i, j, k, s, nullptr);
    if constexpr (ZERO) {
      const T z0 = T(0);
      x[id] = (T(b[id]) - nb_sum<T>(s, z0, z0, z0, z0, z0, z0, nd)) / s.c;
    } else {
      const T zp = D == 3 ? x[id + g.sxy] : T(0);
      const T zm = D == 3 ? x[id - g.sxy] : T(0);
      const T bv = T(b[id]);
      const T v = (bv - nb_sum<T>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, nd)) / s.c;
      x[id] = v;
      if constexpr (DOT) acc += double(bv) * double(v);
    }
  }
}

// One red-black Gauss-Seidel colour pass on the folded operator; colour of
// (i,j,k) is (i+j+k)&1. The updated colour only reads the other colour, so a
// pass is race free.
// ZERO: the first pass of a sweep from a zero field. Every neighbour value
// is zero, so none is loaded (the arithmetic is that of a pass over a
// zero-filled field, so the bits are the same), and the field need not be
// cleared first: the other colour is written by the next pass before any
// pass reads it, and boundary entries are never written.
// DOT: the sum over the updated nodes of b * (new x) is reduced over the grid
// and handed to `post` (the last two passes of a V-cycle's finest level give
// r.z of preconditioned CG, since b is r there).
template <class Coef, typename T, typename TB, bool ZERO = false, bool DOT = false, class Post = NoPost>
__global__ void __launch_bounds__(kBx* kBy, ZERO || sizeof(T) == 4 ? 4 : 3)
    k_rbgs(GridDev g, Coef cf, const TB* __restrict__ b, T* __restrict__ x, int color, const Ctl* ctl,
           RedSlot slot = RedSlot{}, Post post = Post{}) {
  if (ctl_skip_dep(ctl)) return;
  // with DOT every thread reaches the block reduction at the end
  double acc[1] = {0.0};
  if (g.dim == 3)
    rbgs_columns<3, 0, Coef, T, TB, ZERO, DOT>(g, cf, b, x, color, acc[0]);
  else
    rbgs_columns<2, 2, Coef, T, TB, ZERO, DOT>(g, cf, b, x, color, acc[0]);
  if constexpr (DOT) grid_reduce<1, false>(acc, slot, post);
}

// One full red-black Gauss-Seidel sweep in a single pass (colour `first`
// updated first, then the other), reading x_in and writing x_out (distinct
// buffers). The first colour only reads the other colour's old values
// (x_in); the second colour reads the new first-colour values, which each
// block recomputes on its tile plus a one-node halo and keeps in a 3-plane
// shared-memory ring while marching in z. Halo values are computed from
// x_in only, so every block gets identical numbers and the sweep is race free
// and deterministic. One pass moves x, k and b once: half the traffic of two
// colour passes. zero_in: x_in is identically zero (first sweep of a V-cycle
// level), so it is not read.
template <class Coef, typename T, typename TB>
__device__ __forceinline__ T gs_update(const GridDev& g, const Coef& cf, const TB* __restrict__ b, int i, int j,
                                       int k, long long id, T xp, T xm, T yp, T ym, T zp, T zm) {
  Stencil<T> s = cf.template at<T>(g, id);
  fold_faces<T>(g, i, j, k, s, nullptr);
  return (T(b[id]) - nb_sum<T>(s, xp, xm, yp, ym, zp, zm, g.dim)) / s.c;
}

// Tile of the fused sweep: 64 x 8 columns, each thread owns two adjacent
// x-columns (one of each colour on every plane); a ring of first-colour values
// over the tile plus a one-node halo covers kSlab + 2 planes, and each barrier
// phase handles kSlab planes so many loads are in flight per phase.
constexpr int kFx = 2 * kBx;          // 64 columns
constexpr int kHx = kFx + 2, kHy = kBy + 2;
constexpr int kSlab = 4;
constexpr int kRing = kSlab + 2;
constexpr int kHalo = 2 * kHx + 2 * kBy;  // 148 border cells

template <class Coef, typename T, typename TB>
__global__ void __launch_bounds__(kBx* kBy) k_rbgs_fused(GridDev g, Coef cf, const TB* __restrict__ b,
                                                         const T* __restrict__ xin, T* __restrict__ xout,
                                                         int first, int zero_in, const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  __shared__ T ring[kRing][kHy][kHx];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = tx + kBx * ty;
  const int i0 = blockIdx.x * kFx, j0 = blockIdx.y * kBy;
  int k0, k1;
  column_range(g, k0, k1);
  if (k0 >= k1) return;
  const bool is3 = g.dim == 3;
  const int klo = is3 ? 1 : 0, khi = is3 ? g.nz - 2 : 0;
  auto interior = [&](int ii, int jj, int kk) {
    return ii >= 1 && ii <= g.nx - 2 && jj >= 1 && jj <= g.ny - 2 && kk >= klo && kk <= khi;
  };
  auto X = [&](int ii, int jj, int kk) -> T {
    return zero_in ? T(0) : xin[((long long)kk * g.ny + jj) * g.nx + ii];
  };
  // first-colour update at a node from x_in (0 off the interior)
  auto first_val = [&](int ii, int jj, int kk) -> T {
    if (!interior(ii, jj, kk)) return T(0);
    const long long id = ((long long)kk * g.ny + jj) * g.nx + ii;
    const T zp = is3 ? X(ii, jj, kk + 1) : T(0);
    const T zm = is3 ? X(ii, jj, kk - 1) : T(0);
    return gs_update<Coef, T, TB>(g, cf, b, ii, jj, kk, id, X(ii + 1, jj, kk), X(ii - 1, jj, kk), X(ii, jj + 1, kk),
                                  X(ii, jj - 1, kk), zp, zm);
  };
  auto slot = [&](int p) { return ((p % kRing) + kRing) % kRing; };
  // border cell of this thread (tid < kHalo)
  int hcol = -1, hrow = -1;
  if (tid < kHalo) {
    if (tid < kHx) {
      hcol = tid;
      hrow = 0;
    } else if (tid < 2 * kHx) {
      hcol = tid - kHx;
      hrow = kHy - 1;
    } else if (tid < 2 * kHx + kBy) {
      hcol = 0;
      hrow = 1 + (tid - 2 * kHx);
    } else {
      hcol = kHx - 1;
      hrow = 1 + (tid - 2 * kHx - kBy);
    }
  }
  const int jj = j0 + ty;
  // first colour on plane p for the tile + halo; own first-colour nodes of
  // planes in [k0,k1) are also stored to x_out
  auto first_plane = [&](int p) {
    const int sp = slot(p);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int ii = i0 + 2 * tx + c;
      if (((ii + jj + p) & 1) != first) continue;
      const T v = first_val(ii, jj, p);
      ring[sp][ty + 1][2 * tx + c + 1] = v;
      if (p >= k0 && p < k1 && interior(ii, jj, p)) xout[((long long)p * g.ny + jj) * g.nx + ii] = v;
    }
    if (hcol >= 0) {
      const int gi = i0 - 1 + hcol, gj = j0 - 1 + hrow;
      if (((gi + gj + p) & 1) == first) ring[sp][hrow][hcol] = first_val(gi, gj, p);
    }
  };
  auto second_plane = [&](int q) {
    const int sq = slot(q);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int ii = i0 + 2 * tx + c;
      if (((ii + jj + q) & 1) == first || !interior(ii, jj, q)) continue;
      const int col = 2 * tx + c + 1, row = ty + 1;
      const T zp = is3 ? ring[slot(q + 1)][row][col] : T(0);
      const T zm = is3 ? ring[slot(q - 1)][row][col] : T(0);
      const long long id = ((long long)q * g.ny + jj) * g.nx + ii;
      xout[id] = gs_update<Coef, T, TB>(g, cf, b, ii, jj, q, id, ring[sq][row][col + 1], ring[sq][row][col - 1],
                                        ring[sq][row + 1][col], ring[sq][row - 1][col], zp, zm);
    }
  };
  if (!is3) {
    first_plane(0);
    __syncthreads();
    second_plane(0);
    return;
  }
  first_plane(k0 - 1);
  first_plane(k0);
  for (int q0 = k0; q0 < k1; q0 += kSlab) {
    const int qe = min(q0 + kSlab, k1);
    // first colour for planes q0+1 .. qe (plane qe may lie past the chunk)
#pragma unroll
    for (int s = 1; s <= kSlab; ++s)
      if (q0 + s <= qe) first_plane(q0 + s);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < kSlab; ++s)
      if (q0 + s < qe) second_plane(q0 + s);
    __syncthreads();
  }
}

// ------------------------------------------------------------- full apply

// y = L x with identity boundary rows: LinearOperator2D::Apply
// (src/backends/cpu/cpu_utils.cpp:324-513) extended to 3D; optional fused
// sum(w*y).
template <class Coef, int NV, class Post>
__global__ void __launch_bounds__(kBx* kBy) k_apply_full(GridDev g, Coef cf, const double* __restrict__ x,
                                                         double* __restrict__ y, RedSlot slot, Post post,
                                                         const Ctl* ctl, const double* __restrict__ w = nullptr) {
  if (ctl_stopped(ctl)) return;
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  // full z range (boundary planes included) split into chunks
  const int chunk = (g.nz + gridDim.z - 1) / gridDim.z;
  const int k0 = blockIdx.z * chunk, k1 = min(g.nz, k0 + chunk);
  double acc[(NV > 0 ? NV : 1)] = {0.0};
  if (i < g.nx && j < g.ny) {
    for (int k = k0; k < k1; ++k) {
      const long long id = ((long long)k * g.ny + j) * g.nx + i;
      const bool interior = i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2 &&
                            (g.dim == 2 || (k >= 1 && k <= g.nz - 2));
      double v;
      if (interior) {
        const Stencil<double> s = cf.template at<double>(g, id);
        const double zp = g.dim == 3 ? x[id + g.sxy] : 0.0;
        const double zm = g.dim == 3 ? x[id - g.sxy] : 0.0;
        v = s.c * x[id] + nb_sum<double>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, g.dim);
      } else {
        v = x[id];
      }
      y[id] = v;
      if constexpr (NV > 0) acc[0] += (w ? w[id] : x[id]) * v;
    }
  }
  if constexpr (NV > 0) grid_reduce<(NV > 0 ? NV : 1), false>(acc, slot, post);
}

// ---------------------------------------------------------------- Jacobi

// One Jacobi sweep of the reference (relaxation.cpp:426-546, solver.cpp:808-962):
// next = (-(f + nonlinear(u)) - lap)/center on interior nodes, reading the
// stored face values of `grid`; fused max|du| (the reference's stopping
// quantity).
template <class Coef, class Post>
__global__ void __launch_bounds__(kBx* kBy) k_jacobi(GridDev g, Coef cf, const double* __restrict__ f,
                                                     double f_const, NonlinDev nl, const double* __restrict__ grid,
                                                     double* __restrict__ next, RedSlot slot, Post post,
                                                     const Ctl* ctl, int* degenerate) {
  if (ctl_stopped(ctl)) return;
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(g, k0, k1);
  double acc[1] = {0.0};
  if (i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) {
    for (int k = k0; k < k1; ++k) {
      const long long id = ((long long)k * g.ny + j) * g.nx + i;
      const Stencil<double> s = cf.template at<double>(g, id);
      if (fabs(s.c) < 1e-12) {
        *degenerate = 1;
        continue;
      }
      const double zp = g.dim == 3 ? grid[id + g.sxy] : 0.0;
      const double zm = g.dim == 3 ? grid[id - g.sxy] : 0.0;
      const double lap = nb_sum<double>(s, grid[id + 1], grid[id - 1], grid[id + g.nx], grid[id - g.nx], zp, zm, g.dim);
      const double old_u = grid[id];
      const double rhs = -f_plus_nl(f ? f[id] : f_const, nl, old_u) - lap;
      const double upd = __ddiv_rn(rhs, s.c);
      next[id] = upd;
      acc[0] = fmax(acc[0], fabs(upd - old_u));
    }
  }
  grid_reduce<1, true>(acc, slot, post);
}

// -------------------------------------------------------- boundary fill

// Final value of boundary node (i,j,k) after the reference's closure
// sequence Dirichlet / Neumann-Robin (x faces, y faces, z faces) / Dirichlet
// (src/backends/cpu/solver.cpp:751-753, cpu_utils.cpp:575-901):
//  - a node on a Dirichlet face takes the value of the last Dirichlet face
//    written (z over y over x, max over min);
//  - otherwise the last Neumann/Robin phase containing it writes
//    closure(u[inward neighbour]); the inward neighbour is either interior or a
//    boundary node finalised by an earlier phase, so the chain is evaluated
//    from the interior outwards (depth <= 3). Only interior nodes are read,
//    so one launch over all faces is race free.
__device__ __forceinline__ double closure_value(const FaceDev& f, int is_max, int loc, double unb,
                                                bool* ok) {
  *ok = true;
  if (f.kind == kNeumann) {
    const double gv = f.val.at(loc);
    return is_max ? unb + f.h * gv : unb - f.h * gv;
  }
  const double alpha = f.alpha.at(loc), beta = f.beta.at(loc), gamma = f.gamma.at(loc);
  if (!is_max) {
    const double denom = alpha + beta / f.h;
    if (fabs(denom) > 1e-12) return (gamma + (beta / f.h) * unb) / denom;
  } else {
    const double denom = alpha - beta / f.h;
    if (fabs(denom) > 1e-12) return (gamma - (beta / f.h) * unb) / denom;
  }
  *ok = false;
  return 0.0;
}

__device__ __forceinline__ int face_loc(const GridDev& g, int f, int i, int j, int k) {
  return f <= kRight ? j + g.ny * k : (f <= kTop ? i + g.nx * k : i + g.nx * j);
}

// dirichlet_last: the reference sequence ends with its Dirichlet pass (every
// path except 2D Gauss-Seidel/SOR, which applies Dirichlet once before the
// first sweep and only Neumann/Robin closures per iteration,
// relaxation.cpp:66,135). Without it, a node on both kinds of face keeps the
// Neumann/Robin value and a chain may end on a Dirichlet node.
__device__ __forceinline__ double boundary_final(const GridDev& g, const double* u, int i, int j, int k,
                                                 bool dirichlet_last = true) {
  auto dirichlet_winner = [&](int ci, int cj, int ck, double* v) {
    const bool on[6] = {ci == 0, ci == g.nx - 1, cj == 0, cj == g.ny - 1, g.dim == 3 && ck == 0,
                        g.dim == 3 && ck == g.nz - 1};
    for (int f = 5; f >= 0; --f)
      if (on[f] && g.face[f].active && g.face[f].kind == kDirichlet) {
        *v = g.face[f].val.at(face_loc(g, f, ci, cj, ck));
        return true;
      }
    return false;
  };
  double dv;
  if (dirichlet_last && dirichlet_winner(i, j, k, &dv)) return dv;
  int chain_f[3], chain_loc[3], cnt = 0;
  int ci = i, cj = j, ck = k;
  double base = 0.0;
  for (int depth = 0; depth < 4; ++depth) {
    const bool cb[6] = {ci == 0, ci == g.nx - 1, cj == 0, cj == g.ny - 1, g.dim == 3 && ck == 0,
                        g.dim == 3 && ck == g.nz - 1};
    // the last Neumann/Robin phase containing the node writes it
    int f = -1;
    for (int q = 5; q >= 0; --q)
      if (cb[q] && g.face[q].active && g.face[q].kind != kDirichlet) {
        f = q;
        break;
      }
    if (f < 0) {
      const bool bd = cb[0] || cb[1] || cb[2] || cb[3] || cb[4] || cb[5];
      if (bd && dirichlet_winner(ci, cj, ck, &dv))
        base = dv;
      else
        base = u[((long long)ck * g.ny + cj) * g.nx + ci];
      break;
    }
    chain_f[cnt] = f;
    chain_loc[cnt] = face_loc(g, f, ci, cj, ck);
    ++cnt;
    if (f == kLeft) ci = 1;
    else if (f == kRight) ci = g.nx - 2;
    else if (f == kBottom) cj = 1;
    else if (f == kTop) cj = g.ny - 2;
    else if (f == kFront) ck = 1;
    else ck = g.nz - 2;
  }
  double v = base;
  for (int m = cnt - 1; m >= 0; --m) {
    bool ok;
    const double nv = closure_value(g.face[chain_f[m]], chain_f[m] & 1, chain_loc[m], v, &ok);
    if (!ok) return u[((long long)k * g.ny + j) * g.nx + i];  // |denominator| <= 1e-12: node kept
    v = nv;
  }
  return v;
}

// One thread per node of the six faces; a node shared by faces is written by
// the first face (in face order) that contains it.
static __global__ void k_fill_boundary(GridDev g, double* __restrict__ u, const Ctl* ctl, int dirichlet_last = 1) {
  if (ctl_skip(ctl)) return;
  const long long nxy = (long long)g.nx * g.ny;
  const long long nyz = (long long)g.ny * g.nz, nxz = (long long)g.nx * g.nz;
  const long long total = 2 * nyz + 2 * nxz + (g.dim == 3 ? 2 * nxy : 0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
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
    // ownership: the first face in face order containing the node
    const bool on[6] = {i == 0, i == g.nx - 1, j == 0, j == g.ny - 1, g.dim == 3 && k == 0,
                        g.dim == 3 && k == g.nz - 1};
    int owner = -1;
    for (int q = 0; q < 6; ++q)
      if (on[q]) {
        owner = q;
        break;
      }
    if (owner != f) continue;
    u[((long long)k * g.ny + j) * g.nx + i] = boundary_final(g, u, i, j, k, dirichlet_last != 0);
  }
}

// ------------------------------------------------------------ 1D vectors

__device__ __forceinline__ long long gtid() { return blockIdx.x * (long long)blockDim.x + threadIdx.x; }
__device__ __forceinline__ long long gstride() { return (long long)gridDim.x * blockDim.x; }

// x += alpha p ; r -= alpha q ; |r|^2   (alpha = ctl->alpha)
template <typename T, class Post>
__global__ void k_cg_xr(long long n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                        const T* __restrict__ q, RedSlot slot, Post post, Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const double a = ctl->alpha;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    x[t] = T(double(x[t]) + a * double(p[t]));
    const T rv = T(double(r[t]) - a * double(q[t]));
    r[t] = rv;
    acc[0] += double(rv) * double(rv);
  }
  grid_reduce<1, false>(acc, slot, post);
}

// p = z + beta p (beta = ctl->beta; first iteration: p = z)
template <typename T>
__global__ void k_cg_p(long long n, T* __restrict__ p, const T* __restrict__ z, const Ctl* ctl, int first) {
  if (ctl_skip_dep(ctl)) return;
  const double bta = first ? 0.0 : ctl->beta;
  for (long long t = gtid(); t < n; t += gstride()) p[t] = first ? z[t] : T(double(z[t]) + bta * double(p[t]));
}

// sum(a*b) with post
template <typename T, class Post>
__global__ void k_dot(long long n, const T* __restrict__ a, const T* __restrict__ b, RedSlot slot, Post post,
                      const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  double acc[1] = {0.0};
  for (long long t = gtid(); t < n; t += gstride()) acc[0] += double(a[t]) * double(b[t]);
  grid_reduce<1, false>(acc, slot, post);
}

// two dots at once: sum(a*b), sum(c*d)
template <typename T, class Post>
__global__ void k_dot2(long long n, const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ c,
                       const T* __restrict__ d, RedSlot slot, Post post, const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  double acc[2] = {0.0, 0.0};
  for (long long t = gtid(); t < n; t += gstride()) {
    acc[0] += double(a[t]) * double(b[t]);
    acc[1] += double(c[t]) * double(d[t]);
  }
  grid_reduce<2, false>(acc, slot, post);
}

template <typename TD, typename TS>
__global__ void k_convert(long long n, TD* __restrict__ dst, const TS* __restrict__ src) {
  for (long long t = gtid(); t < n; t += gstride()) dst[t] = TD(src[t]);
}

template <typename T>
__global__ void k_fill(long long n, T* __restrict__ dst, T v, const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  for (long long t = gtid(); t < n; t += gstride()) dst[t] = v;
}

// ------------------------------------------------------------ multigrid

// Homogeneous closure chain of a boundary node: the folded system eliminates
// boundary node b through u_b = c0 + c1*u_inward, applied in the reference's
// phase order (x, y, z faces; the last phase containing b writes it). For a
// correction field (c0 = 0) the value at b is coef * u(end), where `end` is the
// interior node the chain reaches. Nodes on a Dirichlet face have coef 0.
// (i,j,k) is moved to `end`; returns coef.
__device__ __forceinline__ double ext_chain(const GridDev& g, int& i, int& j, int& k) {
  {
    const bool on[6] = {i == 0, i == g.nx - 1, j == 0, j == g.ny - 1, g.dim == 3 && k == 0,
                        g.dim == 3 && k == g.nz - 1};
    for (int f = 0; f < 6; ++f)
      if (on[f] && g.face[f].active && g.face[f].kind == kDirichlet) return 0.0;
  }
  double coef = 1.0;
  for (int depth = 0; depth < 3; ++depth) {
    int f = -1;
    if (g.dim == 3 && k == g.nz - 1) f = kBack;
    else if (g.dim == 3 && k == 0) f = kFront;
    else if (j == g.ny - 1) f = kTop;
    else if (j == 0) f = kBottom;
    else if (i == g.nx - 1) f = kRight;
    else if (i == 0) f = kLeft;
    if (f < 0) break;
    const int loc = f <= kRight ? j + g.ny * k : (f <= kTop ? i + g.nx * k : i + g.nx * j);
    coef *= g.face[f].c1.at(loc);
    if (f == kLeft) i = 1;
    else if (f == kRight) i = g.nx - 2;
    else if (f == kBottom) j = 1;
    else if (f == kTop) j = g.ny - 2;
    else if (f == kFront) k = 1;
    else k = g.nz - 2;
  }
  return coef;
}

__device__ __forceinline__ long long cidx(const GridDev& g, int i, int j, int k) {
  return ((long long)k * g.ny + j) * g.nx + i;
}

// Transfer maps for any fine/coarse pair n -> nc per dimension: coarse node I
// sits at fine position I*(n-1)/(nc-1). Three forms, chosen per dimension:
// identity (nc = n, semi-coarsening), nested 2:1 (n odd, nc = (n+1)/2) and
// general (n even, nc = n/2 + 1). The nested form is the general formula
// evaluated exactly (weights 1/2 and 1/4 are exact), so the forms agree bit
// for bit where they overlap.
__device__ __forceinline__ int map_mode(int n, int nc) { return nc == n ? 0 : (2 * nc - 1 == n ? 1 : 2); }

// Interpolation position of fine node i: coarse interval I0 and weight t of
// node I0 + 1 (t = 0 on coincident nodes).
__device__ __forceinline__ void coarse_pos(int i, int n, int nc, int mode, int& I0, double& t) {
  if (mode == 0) {
    I0 = i;
    t = 0.0;
    return;
  }
  if (mode == 1) {
    I0 = i >> 1;
    t = (i & 1) ? 0.5 : 0.0;
    return;
  }
  const int num = i * (nc - 1);
  I0 = num / (n - 1);
  const int rem = num - I0 * (n - 1);
  t = double(rem) / double(n - 1);
  if (I0 >= nc - 1) {
    I0 = nc - 1;
    t = 0.0;
  }
}

// Restriction weights of coarse node I over fine nodes, the scaled transpose
// of the interpolation: w_i = (nc-1)/(n-1) * max(0, 1 - |i(nc-1) - I(n-1)|/(n-1))
// ({1/4, 1/2, 1/4} for the nested form). Always four consecutive entries
// (i0 .. i0+3); entries outside the grid or the support carry weight 0 and a
// clamped index.
__device__ __forceinline__ void restrict_weights(int I, int n, int nc, int mode, int& i0, double (&w)[4]) {
  if (mode == 0) {
    i0 = I;
    w[0] = 1.0;
    w[1] = w[2] = w[3] = 0.0;
    return;
  }
  if (mode == 1) {
    i0 = 2 * I - 1;
    w[0] = 0.25;
    w[1] = 0.5;
    w[2] = 0.25;
    w[3] = 0.0;
  } else {
    const int den = n - 1, m = nc - 1;
    const int num = (I - 1) * den;
    const int fl = num >= 0 ? num / m : -((-num + m - 1) / m);
    i0 = fl + 1;
    const double scale = double(m) / double(den);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int d = (i0 + q) * m - I * den;
      d = d < 0 ? -d : d;
      w[q] = d < den ? scale * (1.0 - double(d) / double(den)) : 0.0;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (i0 + q < 0 || i0 + q > n - 1) w[q] = 0.0;
}

__device__ __forceinline__ int clampi(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Full weighting of the fine residual at coarse node (I,J,K), boundary coarse
// nodes included (fine boundary values of the residual are zero).
template <typename T>
__device__ __forceinline__ double full_weight(const GridDev& gf, const GridDev& gc, const T* __restrict__ rf, int I,
                                              int J, int K) {
  int ix0, iy0, iz0 = 0;
  double wx[4], wy[4], wz[4] = {1.0, 0.0, 0.0, 0.0};
  restrict_weights(I, gf.nx, gc.nx, map_mode(gf.nx, gc.nx), ix0, wx);
  restrict_weights(J, gf.ny, gc.ny, map_mode(gf.ny, gc.ny), iy0, wy);
  const bool is3 = gc.dim == 3;
  if (is3) restrict_weights(K, gf.nz, gc.nz, map_mode(gf.nz, gc.nz), iz0, wz);
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (wz[c] == 0.0) continue;
    const long long plane = (long long)clampi(iz0 + c, gf.nz - 1) * gf.ny;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (wy[b] == 0.0) continue;
      const T* row = rf + (plane + clampi(iy0 + b, gf.ny - 1)) * gf.nx;
      double rs = 0.0;
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (wx[a] != 0.0) rs += wx[a] * double(row[clampi(ix0 + a, gf.nx - 1)]);
      acc += wz[c] * wy[b] * rs;
    }
  }
  return acc;
}

// Restriction R = Ext^T P^T / 2^dim, in two race-free launches:
//  k_restrict_fw   full weighting of the fine residual at every coarse node,
//                  boundary nodes included (one thread per coarse node);
//  k_restrict_fold_faces  interior coarse nodes next to a Neumann/Robin face
//                  add coef * value of each boundary node whose closure chain
//                  ends at them (the transpose of the extended prolongation
//                  below).
// Boundary entries of the coarse right-hand side are left holding their full
// weights; no coarse kernel reads them.
template <typename T, typename TC>
__global__ void __launch_bounds__(kBx* kBy) k_restrict_fw(GridDev gf, GridDev gc, const T* __restrict__ rf,
                                                          TC* __restrict__ bc, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const int I = blockIdx.x * kBx + threadIdx.x;
  const int J = blockIdx.y * kBy + threadIdx.y;
  if (I >= gc.nx || J >= gc.ny) return;
  const int chunk = (gc.nz + gridDim.z - 1) / gridDim.z;
  const int K0 = blockIdx.z * chunk, K1 = min(gc.nz, K0 + chunk);
  for (int K = K0; K < K1; ++K) bc[cidx(gc, I, J, K)] = TC(full_weight<T>(gf, gc, rf, I, J, K));
}

// The fold on the face-adjacent interior coarse nodes, one thread per node:
// the nodes are enumerated layer by layer (i = 1, i = nx-2, j = 1, j = ny-2,
// k = 1, k = nz-2), each layer without the nodes of the layers before it, so
// every node is visited once; reads go to boundary nodes only and writes to
// interior nodes only, so one launch is race free.
struct FoldLayers {
  long long start[7];  // prefix counts of the six layers
};

inline FoldLayers fold_layers(const GridDev& g) {
  FoldLayers L{};
  const long long ni = g.nx - 2, nj = g.ny - 2, nk = g.dim == 3 ? g.nz - 2 : 1;
  const long long mi = ni > 2 ? ni - 2 : 0, mj = nj > 2 ? nj - 2 : 0;  // i (j) not on an x (y) layer
  long long c[6];
  c[0] = nj * nk;                               // i = 1
  c[1] = ni > 1 ? nj * nk : 0;                  // i = nx-2
  c[2] = mi * nk;                               // j = 1
  c[3] = nj > 1 ? mi * nk : 0;                  // j = ny-2
  c[4] = g.dim == 3 ? mi * mj : 0;              // k = 1
  c[5] = g.dim == 3 && nk > 1 ? mi * mj : 0;    // k = nz-2
  L.start[0] = 0;
  for (int q = 0; q < 6; ++q) L.start[q + 1] = L.start[q] + c[q];
  return L;
}

template <typename TC>
__global__ void __launch_bounds__(256) k_restrict_fold_faces(GridDev gc, FoldLayers lay, TC* __restrict__ bc,
                                                             const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const long long ni = gc.nx - 2, nj = gc.ny - 2;
  const long long mi = ni > 2 ? ni - 2 : 0;
  const int kb = gc.dim == 3 ? 1 : 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < lay.start[6];
       t += (long long)gridDim.x * blockDim.x) {
    int q = 0;
    while (t >= lay.start[q + 1]) ++q;
    const long long u = t - lay.start[q];
    int I, J, K;
    if (q <= 1) {  // x layers: all interior (j, k)
      I = q == 0 ? 1 : gc.nx - 2;
      J = 1 + int(u % nj);
      K = kb + int(u / nj);
    } else if (q <= 3) {  // y layers: i off the x layers, all interior k
      J = q == 2 ? 1 : gc.ny - 2;
      I = 2 + int(u % mi);
      K = kb + int(u / mi);
    } else {  // z layers: i and j off the x and y layers
      K = q == 4 ? 1 : gc.nz - 2;
      I = 2 + int(u % mi);
      J = 2 + int(u / mi);
    }
    const int dxl = I == 1 ? -1 : 0, dxh = I == gc.nx - 2 ? 1 : 0;
    const int dyl = J == 1 ? -1 : 0, dyh = J == gc.ny - 2 ? 1 : 0;
    const int dzl = gc.dim == 3 && K == 1 ? -1 : 0, dzh = gc.dim == 3 && K == gc.nz - 2 ? 1 : 0;
    double acc = 0.0;
    for (int dk = dzl; dk <= dzh; ++dk)
      for (int dj = dyl; dj <= dyh; ++dj)
        for (int di = dxl; di <= dxh; ++di) {
          if (di == 0 && dj == 0 && dk == 0) continue;
          int ci = I + di, cj = J + dj, ck = K + dk;
          const double coef = ext_chain(gc, ci, cj, ck);
          if (coef != 0.0 && ci == I && cj == J && ck == K) acc += coef * double(bc[cidx(gc, I + di, J + dj, K + dk)]);
        }
    if (acc != 0.0) {
      const long long id = cidx(gc, I, J, K);
      bc[id] = TC(double(bc[id]) + acc);
    }
  }
}

// coarse correction value at any coarse node, boundary nodes by the
// homogeneous closure chain
template <typename TC>
__device__ __forceinline__ double ext_value(const GridDev& gc, const TC* __restrict__ xc, int I, int J, int K) {
  const bool bd = I == 0 || I == gc.nx - 1 || J == 0 || J == gc.ny - 1 || (gc.dim == 3 && (K == 0 || K == gc.nz - 1));
  if (!bd) return double(xc[cidx(gc, I, J, K)]);
  const double coef = ext_chain(gc, I, J, K);
  return coef == 0.0 ? 0.0 : coef * double(xc[cidx(gc, I, J, K)]);
}

// Trilinear (bilinear in 2D) interpolation of the coarse correction, extended
// to the coarse boundary through the closures, added to the fine interior.
template <typename T, typename TC>
__global__ void __launch_bounds__(kBx* kBy) k_prolong_add(GridDev gf, GridDev gc, const TC* __restrict__ xc,
                                                          T* __restrict__ xf, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(gf, k0, k1);
  if (!(i >= 1 && i <= gf.nx - 2 && j >= 1 && j <= gf.ny - 2)) return;
  int I0, J0;
  double tx, ty;
  coarse_pos(i, gf.nx, gc.nx, map_mode(gf.nx, gc.nx), I0, tx);
  coarse_pos(j, gf.ny, gc.ny, map_mode(gf.ny, gc.ny), J0, ty);
  const int I1 = tx != 0.0 ? I0 + 1 : I0, J1 = ty != 0.0 ? J0 + 1 : J0;
  const bool xy_edge = I0 == 0 || I1 == gc.nx - 1 || J0 == 0 || J1 == gc.ny - 1;
  const int zmode = gf.dim == 3 ? map_mode(gf.nz, gc.nz) : 0;
  for (int k = k0; k < k1; ++k) {
    int K0 = 0, K1 = 0;
    double tz = 0.0;
    if (gf.dim == 3) {
      coarse_pos(k, gf.nz, gc.nz, zmode, K0, tz);
      K1 = tz != 0.0 ? K0 + 1 : K0;
    }
    double c000, c100, c010, c110, c001, c101, c011, c111;
    if (!xy_edge && !(gf.dim == 3 && (K0 == 0 || K1 == gc.nz - 1))) {
      const long long a0 = (long long)K0 * gc.sxy, a1 = (long long)K1 * gc.sxy;
      const long long r0 = (long long)J0 * gc.nx, r1 = (long long)J1 * gc.nx;
      c000 = double(xc[a0 + r0 + I0]);
      c100 = double(xc[a0 + r0 + I1]);
      c010 = double(xc[a0 + r1 + I0]);
      c110 = double(xc[a0 + r1 + I1]);
      c001 = double(xc[a1 + r0 + I0]);
      c101 = double(xc[a1 + r0 + I1]);
      c011 = double(xc[a1 + r1 + I0]);
      c111 = double(xc[a1 + r1 + I1]);
    } else {
      c000 = ext_value(gc, xc, I0, J0, K0);
      c100 = ext_value(gc, xc, I1, J0, K0);
      c010 = ext_value(gc, xc, I0, J1, K0);
      c110 = ext_value(gc, xc, I1, J1, K0);
      c001 = ext_value(gc, xc, I0, J0, K1);
      c101 = ext_value(gc, xc, I1, J0, K1);
      c011 = ext_value(gc, xc, I0, J1, K1);
      c111 = ext_value(gc, xc, I1, J1, K1);
    }
    const double x00 = (1.0 - tx) * c000 + tx * c100, x10 = (1.0 - tx) * c010 + tx * c110;
    const double x01 = (1.0 - tx) * c001 + tx * c101, x11 = (1.0 - tx) * c011 + tx * c111;
    const double y0 = (1.0 - ty) * x00 + ty * x10, y1 = (1.0 - ty) * x01 + ty * x11;
    const double v = (1.0 - tz) * y0 + tz * y1;
    const long long id = ((long long)k * gf.ny + j) * gf.nx + i;
    xf[id] = T(double(xf[id]) + v);
  }
}

// z-marching transfer kernels for level pairs whose z map is the identity or
// nested 2:1 (every odd side, and every 2D grid). One thread per column:
// restriction sums each fine plane's x-y weights once and shares the plane
// sum between the two coarse planes it feeds; prolongation evaluates the
// bilinear x-y interpolation once per coarse plane and reuses it for the 2-3
// fine planes it feeds (same expressions as k_prolong_add, so the same bits).
__device__ __forceinline__ bool z_marchable(const GridDev& gf, const GridDev& gc) {
  return gf.dim != 3 || map_mode(gf.nz, gc.nz) <= 1;
}

// Full weighting of one coarse column (I, J): the x-y weights once, then the
// weighted sum of any fine plane.
template <typename T>
struct FwColumn {
  const T* rf;
  int nx, ny, ix0, iy0;
  double wx[4], wy[4];
  __device__ __forceinline__ void init(const GridDev& gf, const GridDev& gc, const T* r, int I, int J) {
    rf = r;
    nx = gf.nx;
    ny = gf.ny;
    restrict_weights(I, gf.nx, gc.nx, map_mode(gf.nx, gc.nx), ix0, wx);
    restrict_weights(J, gf.ny, gc.ny, map_mode(gf.ny, gc.ny), iy0, wy);
  }
  // Interior column of a nested 2:1 map in x and y: taps (1/4, 1/2, 1/4) at
  // 2I-1..2I+1 and 2J-1..2J+1, all in range. Same operations in the same
  // order as plane(), without the weight tests, so all nine loads can be
  // issued together.
  __device__ __forceinline__ double plane_nested(int kf) const {
    double acc = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const T* row = rf + ((long long)kf * ny + (iy0 + b)) * nx + ix0;
      double rs = 0.0;
      rs += 0.25 * double(row[0]);
      rs += 0.5 * double(row[1]);
      rs += 0.25 * double(row[2]);
      acc += (b == 1 ? 0.5 : 0.25) * rs;
    }
    return acc;
  }
  __device__ __forceinline__ double plane(int kf) const {
    double acc = 0.0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      if (wy[b] == 0.0) continue;
      const T* row = rf + ((long long)kf * ny + clampi(iy0 + b, ny - 1)) * nx;
      double rs = 0.0;
#pragma unroll
      for (int a = 0; a < 4; ++a)
        if (wx[a] != 0.0) rs += wx[a] * double(row[clampi(ix0 + a, nx - 1)]);
      acc += wy[b] * rs;
    }
    return acc;
  }
};

template <typename T, typename TC>
__global__ void __launch_bounds__(kBx* kBy) k_restrict_march(GridDev gf, GridDev gc, const T* __restrict__ rf,
                                                             TC* __restrict__ bc, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const int I = blockIdx.x * kBx + threadIdx.x;
  const int J = blockIdx.y * kBy + threadIdx.y;
  if (I >= gc.nx || J >= gc.ny) return;
  const int chunk = (gc.nz + gridDim.z - 1) / gridDim.z;
  const int K0 = blockIdx.z * chunk, K1 = min(gc.nz, K0 + chunk);
  FwColumn<T> col;
  col.init(gf, gc, rf, I, J);
  const bool nested = map_mode(gf.nx, gc.nx) == 1 && map_mode(gf.ny, gc.ny) == 1 && I >= 1 && I <= gc.nx - 2 &&
                      J >= 1 && J <= gc.ny - 2;
  auto plane = [&](int kf) -> double { return nested ? col.plane_nested(kf) : col.plane(kf); };
  const long long cxy = (long long)J * gc.nx + I;
  if (gc.dim != 3 || gc.nz == gf.nz) {
    for (int K = K0; K < K1; ++K) bc[(long long)K * gc.sxy + cxy] = TC(plane(K));
    return;
  }
  // nested 2:1 in z: coarse K takes fine planes 2K-1, 2K, 2K+1 with 1/4, 1/2, 1/4
  double below = 2 * K0 - 1 >= 0 ? plane(2 * K0 - 1) : 0.0;
#pragma unroll 2
  for (int K = K0; K < K1; ++K) {
    const double mid = plane(2 * K);
    const double above = 2 * K + 1 <= gf.nz - 1 ? plane(2 * K + 1) : 0.0;
    bc[(long long)K * gc.sxy + cxy] = TC(0.25 * below + 0.5 * mid + 0.25 * above);
    below = above;
  }
}

template <typename T, typename TC>
__global__ void __launch_bounds__(kBx* kBy) k_prolong_march(GridDev gf, GridDev gc, const TC* __restrict__ xc,
                                                            T* __restrict__ xf, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const int i = blockIdx.x * kBx + threadIdx.x;
  const int j = blockIdx.y * kBy + threadIdx.y;
  int k0, k1;
  column_range(gf, k0, k1);
  if (!(i >= 1 && i <= gf.nx - 2 && j >= 1 && j <= gf.ny - 2) || k0 >= k1) return;
  int I0, J0;
  double tx, ty;
  coarse_pos(i, gf.nx, gc.nx, map_mode(gf.nx, gc.nx), I0, tx);
  coarse_pos(j, gf.ny, gc.ny, map_mode(gf.ny, gc.ny), J0, ty);
  const int I1 = tx != 0.0 ? I0 + 1 : I0, J1 = ty != 0.0 ? J0 + 1 : J0;
  const bool xy_edge = I0 == 0 || I1 == gc.nx - 1 || J0 == 0 || J1 == gc.ny - 1;
  const int zmode = gf.dim == 3 ? map_mode(gf.nz, gc.nz) : 0;
  // bilinear value on coarse plane K (boundary values through the closures)
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
  // groups of four planes: the four fine values are loaded before any is
  // stored, so a thread has four loads in flight instead of one
  constexpr int kGroup = 4;
  for (int kg = k0; kg < k1; kg += kGroup) {
    T old[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; ++q)
      if (kg + q < k1) old[q] = xf[((long long)(kg + q) * gf.ny + j) * gf.nx + i];
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const int k = kg + q;
      if (k >= k1) break;
      int K0 = 0;
      double tz = 0.0;
      if (gf.dim == 3) coarse_pos(k, gf.nz, gc.nz, zmode, K0, tz);
      const double y0 = at(K0);
      const double y1 = tz != 0.0 ? at(K0 + 1) : y0;
      const double v = (1.0 - tz) * y0 + tz * y1;
      xf[((long long)k * gf.ny + j) * gf.nx + i] = T(double(old[q]) + v);
    }
  }
}

// Prolongation-add for a level pair nested 2:1 in x, y and z (3D): a thread
// owns coarse column (I, J) and the four fine columns 2I+a, 2J+b (a, b = 0, 1)
// it interpolates to, and marches over a chunk of coarse planes K, writing fine
// planes 2K and 2K+1. The four coarse values of a plane are loaded once for
// the four columns, and the eight fine values of a step are loaded before
// any is stored; the arithmetic of every fine node is that of
// k_prolong_march (same weights and expressions, so the same bits). At 257^3:
// 68 against 98.5 us per launch stand-alone.
template <typename T, typename TC>
__global__ void __launch_bounds__(kBx* kBy) k_prolong_pair(GridDev gf, GridDev gc, const TC* __restrict__ xc,
                                                           T* __restrict__ xf, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  const int I = blockIdx.x * kBx + threadIdx.x;
  const int J = blockIdx.y * kBy + threadIdx.y;
  if (I > gc.nx - 2 || J > gc.ny - 2) return;
  const int nK = gc.nz - 1;  // coarse planes K = 0 .. nz_c - 2 carry fine planes 2K, 2K+1
  const int chunk = (nK + gridDim.z - 1) / gridDim.z;
  const int Ka = blockIdx.z * chunk, Kb = min(nK, Ka + chunk);
  if (Ka >= Kb) return;
  const bool xy_edge = I == 0 || I + 1 == gc.nx - 1 || J == 0 || J + 1 == gc.ny - 1;
  // bilinear values of the four fine columns on coarse plane K (boundary
  // values through the closures, as in k_prolong_march)
  auto bil4 = [&](int K, double (&y)[4]) {
    double C00, C10, C01, C11;
    if (!xy_edge && !(K == 0 || K == gc.nz - 1)) {
      const long long a = (long long)K * gc.sxy + (long long)J * gc.nx + I;
      C00 = double(xc[a]);
      C10 = double(xc[a + 1]);
      C01 = double(xc[a + gc.nx]);
      C11 = double(xc[a + gc.nx + 1]);
    } else {
      C00 = ext_value(gc, xc, I, J, K);
      C10 = ext_value(gc, xc, I + 1, J, K);
      C01 = ext_value(gc, xc, I, J + 1, K);
      C11 = ext_value(gc, xc, I + 1, J + 1, K);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int a = q & 1, b = q >> 1;
      const double tx = a ? 0.5 : 0.0, ty = b ? 0.5 : 0.0;
      const double c00 = C00, c10 = a ? C10 : C00, c01 = b ? C01 : C00, c11 = a ? (b ? C11 : C10) : (b ? C01 : C00);
      const double x0 = (1.0 - tx) * c00 + tx * c10, x1 = (1.0 - tx) * c01 + tx * c11;
      y[q] = (1.0 - ty) * x0 + ty * x1;
    }
  };
  double y0[4], y1[4];
  bil4(Ka, y0);
  for (int K = Ka; K < Kb; ++K) {
    bil4(K + 1, y1);
    const int k0 = 2 * K, k1 = 2 * K + 1;
    T old[8];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long c = (long long)(2 * J + (q >> 1)) * gf.nx + 2 * I + (q & 1);
      old[q] = xf[(long long)k0 * gf.sxy + c];
      old[4 + q] = xf[(long long)k1 * gf.sxy + c];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = 2 * I + (q & 1), j = 2 * J + (q >> 1);
      if (i < 1 || j < 1) continue;  // boundary columns of the fine level
      const long long c = (long long)j * gf.nx + i;
      if (k0 >= 1) {
        const double tz = 0.0;
        const double v = (1.0 - tz) * y0[q] + tz * y0[q];
        xf[(long long)k0 * gf.sxy + c] = T(double(old[q]) + v);
      }
      {
        const double tz = 0.5;
        const double v = (1.0 - tz) * y0[q] + tz * y1[q];
        xf[(long long)k1 * gf.sxy + c] = T(double(old[4 + q]) + v);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) y0[q] = y1[q];
  }
}

// Coarse k by injection from the nearest fine node (k_c(I) = k_f(2I) for odd n).
__device__ __forceinline__ int nearest_fine(int I, int n, int nc) {
  return (I * (n - 1) + (nc - 1) / 2) / (nc - 1);
}

template <typename KT>
__global__ void k_inject(GridDev gf, GridDev gc, const KT* __restrict__ kf, KT* __restrict__ kc) {
  for (long long t = gtid(); t < gc.n; t += gstride()) {
    const int I = int(t % gc.nx);
    const int J = int((t / gc.nx) % gc.ny);
    const int K = int(t / gc.sxy);
    const int fi = nearest_fine(I, gf.nx, gc.nx), fj = nearest_fine(J, gf.ny, gc.ny);
    const int fk = gc.dim == 3 ? nearest_fine(K, gf.nz, gc.nz) : 0;
    kc[t] = kf[((long long)fk * gf.ny + fj) * gf.nx + fi];
  }
}

// Coarsest level: `sweeps` red-black GS sweeps from zero, one block.
template <class Coef, typename T, typename TB>
__global__ void k_coarse_solve(GridDev g, Coef cf, const TB* __restrict__ b, T* __restrict__ x, int sweeps,
                               const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  const int tid = threadIdx.x;
  for (long long t = tid; t < g.n; t += blockDim.x) x[t] = T(0);
  __syncthreads();
  const int kb = g.dim == 3 ? 1 : 0, ke = g.dim == 3 ? g.nz - 1 : 1;
  const int ni = g.nx - 2, nj = g.ny - 2, nk = ke - kb;
  const int total = ni * nj * nk;
  for (int s = 0; s < sweeps; ++s) {
    for (int color = 0; color < 2; ++color) {
      for (int t = tid; t < total; t += blockDim.x) {
        const int i = 1 + t % ni, j = 1 + (t / ni) % nj, k = kb + t / (ni * nj);
        if (((i + j + k) & 1) != color) continue;
        const long long id = ((long long)k * g.ny + j) * g.nx + i;
        Stencil<T> st = cf.template at<T>(g, id);
        fold_faces<T>(g, i, j, k, st, nullptr);
        const T zp = g.dim == 3 ? x[id + g.sxy] : T(0);
        const T zm = g.dim == 3 ? x[id - g.sxy] : T(0);
        x[id] = (T(b[id]) - nb_sum<T>(st, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, g.dim)) / st.c;
      }
      __syncthreads();
    }
  }
}

// Coarsest level in shared memory: the folded stencils of all interior nodes
// are evaluated once, then `sweeps` red-black sweeps run on-chip from zero.
// For coarsest grids of at most kCoarseMaxNodes nodes / kCoarseMaxInterior
// interior nodes (checked by the host).
constexpr int kCoarseMaxNodes = 1024;
constexpr int kCoarseMaxInterior = 512;

template <class Coef, typename T, typename TB>
__global__ void k_coarse_solve_smem(GridDev g, Coef cf, const TB* __restrict__ b, T* __restrict__ x, int sweeps,
                                    const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  __shared__ T sx[kCoarseMaxNodes];
  __shared__ T sb[kCoarseMaxInterior];
  __shared__ T sw[kCoarseMaxInterior][7];
  __shared__ int sid[kCoarseMaxInterior];
  const int tid = threadIdx.x;
  const int n = (int)g.n;
  for (int t = tid; t < n; t += blockDim.x) sx[t] = T(0);
  const int kb = g.dim == 3 ? 1 : 0, ke = g.dim == 3 ? g.nz - 1 : 1;
  const int ni = g.nx - 2, nj = g.ny - 2, nk = ke - kb;
  const int total = ni * nj * nk;
  for (int t = tid; t < total; t += blockDim.x) {
    const int i = 1 + t % ni, j = 1 + (t / ni) % nj, k = kb + t / (ni * nj);
    const long long id = ((long long)k * g.ny + j) * g.nx + i;
    Stencil<T> st = cf.template at<T>(g, id);
    fold_faces<T>(g, i, j, k, st, nullptr);
    sw[t][0] = st.c;
    sw[t][1] = st.xp;
    sw[t][2] = st.xm;
    sw[t][3] = st.yp;
    sw[t][4] = st.ym;
    sw[t][5] = st.zp;
    sw[t][6] = st.zm;
    sb[t] = T(b[id]);
    sid[t] = (int)id;
  }
  __syncthreads();
  const int sxy = (int)g.sxy, nx = g.nx;
  if (total == 1) sweeps = sweeps < 1 ? sweeps : 1;  // one interior node: the first sweep is the fixed point
  for (int s = 0; s < sweeps; ++s)
    for (int color = 0; color < 2; ++color) {
      for (int t = tid; t < total; t += blockDim.x) {
        const int i = 1 + t % ni, j = 1 + (t / ni) % nj, k = kb + t / (ni * nj);
        if (((i + j + k) & 1) != color) continue;
        const int id = sid[t];
        T v = sw[t][1] * sx[id + 1] + sw[t][2] * sx[id - 1] + sw[t][3] * sx[id + nx] + sw[t][4] * sx[id - nx];
        if (g.dim == 3) v = v + sw[t][5] * sx[id + sxy] + sw[t][6] * sx[id - sxy];
        sx[id] = (sb[t] - v) / sw[t][0];
      }
      __syncthreads();
    }
  for (int t = tid; t < n; t += blockDim.x) x[t] = sx[t];
}

// ------------------------------------------------------- single-block tail

// The small levels of a V-cycle in one launch. Levels [0, nlev) of `lv` are
// the hierarchy's levels from the first small one down to the coarsest; the
// block runs, with a barrier between phases, exactly the sequence the
// per-level launches run: zero fill and `pre` red-black sweeps, residual,
// full-weighting restriction and boundary fold, recursion, trilinear
// prolongation-add of the extended correction and `post` sweeps (colour order
// reversed), and `coarse_iters` sweeps from zero on the coarsest level. The
// arithmetic of every node update is that of k_rbgs / k_residual_folded /
// full_weight / k_restrict_fold_faces / k_prolong_add. rhs0 is the right-hand side of
// level 0 of the tail; the result is left in lv[0].x.
template <class Coef, typename T>
struct TailLevel {
  GridDev g;
  Coef cf;
  T* x;
  T* b;
  T* r;
};

constexpr int kTailThreads = 512;
constexpr int kTailMaxLevels = 8;

template <class Coef, typename T>
__device__ __forceinline__ void tail_decode(const GridDev& g, int t, int& i, int& j, int& k) {
  const int ni = g.nx - 2, nj = g.ny - 2;
  i = 1 + t % ni;
  j = 1 + (t / ni) % nj;
  k = (g.dim == 3 ? 1 : 0) + t / (ni * nj);
}

template <class Coef, typename T>
__device__ void tail_sweeps(const TailLevel<Coef, T>& L, const T* b, int sweeps, int first) {
  const GridDev& g = L.g;
  const int total = (g.nx - 2) * (g.ny - 2) * (g.dim == 3 ? g.nz - 2 : 1);
  T* x = L.x;
  for (int s = 0; s < sweeps; ++s)
    for (int half = 0; half < 2; ++half) {
      const int color = first ^ half;
      for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int i, j, k;
        tail_decode<Coef, T>(g, t, i, j, k);
        if (((i + j + k) & 1) != color) continue;
        const long long id = ((long long)k * g.ny + j) * g.nx + i;
        Stencil<T> st = L.cf.template at<T>(g, id);
        fold_faces<T>(g, i, j, k, st, nullptr);
        const T zp = g.dim == 3 ? x[id + g.sxy] : T(0);
        const T zm = g.dim == 3 ? x[id - g.sxy] : T(0);
        x[id] = (T(b[id]) - nb_sum<T>(st, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm, g.dim)) / st.c;
      }
      __syncthreads();
    }
}

template <class Coef, typename T>
__device__ void tail_zero(const TailLevel<Coef, T>& L) {
  for (long long t = threadIdx.x; t < L.g.n; t += blockDim.x) L.x[t] = T(0);
  __syncthreads();
}

template <class Coef, typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_tail_vcycle(const TailLevel<Coef, T>* __restrict__ lv, int nlev,
                                                               const T* __restrict__ rhs0, int pre, int post,
                                                               int coarse_iters, int fold, const Ctl* ctl) {
  if (ctl_skip_dep(ctl)) return;
  // down: smooth, residual, restrict
  for (int l = 0; l + 1 < nlev; ++l) {
    const TailLevel<Coef, T>& L = lv[l];
    const T* b = l == 0 ? rhs0 : L.b;
    const GridDev& g = L.g;
    tail_zero(L);
    tail_sweeps(L, b, pre, 0);
    const int total = (g.nx - 2) * (g.ny - 2) * (g.dim == 3 ? g.nz - 2 : 1);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int i, j, k;
      tail_decode<Coef, T>(g, t, i, j, k);
      const long long id = ((long long)k * g.ny + j) * g.nx + i;
      Stencil<T> s = L.cf.template at<T>(g, id);
      fold_faces<T>(g, i, j, k, s, nullptr);
      const T* x = L.x;
      const T zp = g.dim == 3 ? x[id + g.sxy] : T(0);
      const T zm = g.dim == 3 ? x[id - g.sxy] : T(0);
      L.r[id] = T(b[id]) - (s.c * x[id] + nb_sum<T>(s, x[id + 1], x[id - 1], x[id + g.nx], x[id - g.nx], zp, zm,
                                                    g.dim));
    }
    __syncthreads();
    const TailLevel<Coef, T>& C = lv[l + 1];
    const GridDev& gc = C.g;
    for (long long t = threadIdx.x; t < gc.n; t += blockDim.x) {
      const int I = int(t % gc.nx), J = int((t / gc.nx) % gc.ny), K = int(t / gc.sxy);
      C.b[t] = T(full_weight<T>(g, gc, L.r, I, J, K));
    }
    __syncthreads();
    if (fold) {
      const int ctotal = (gc.nx - 2) * (gc.ny - 2) * (gc.dim == 3 ? gc.nz - 2 : 1);
      // each interior coarse node next to a face gathers the boundary values
      // whose closure chain ends at it; writes go to interior nodes only and
      // reads to boundary nodes only, so one pass is race free
      for (int t = threadIdx.x; t < ctotal; t += blockDim.x) {
        int I, J, K;
        tail_decode<Coef, T>(gc, t, I, J, K);
        const int dxl = I == 1 ? -1 : 0, dxh = I == gc.nx - 2 ? 1 : 0;
        const int dyl = J == 1 ? -1 : 0, dyh = J == gc.ny - 2 ? 1 : 0;
        const int dzl = gc.dim == 3 && K == 1 ? -1 : 0, dzh = gc.dim == 3 && K == gc.nz - 2 ? 1 : 0;
        if (dxl == 0 && dxh == 0 && dyl == 0 && dyh == 0 && dzl == 0 && dzh == 0) continue;
        double acc = 0.0;
        for (int dk = dzl; dk <= dzh; ++dk)
          for (int dj = dyl; dj <= dyh; ++dj)
            for (int di = dxl; di <= dxh; ++di) {
              if (di == 0 && dj == 0 && dk == 0) continue;
              int ci = I + di, cj = J + dj, ck = K + dk;
              const double coef = ext_chain(gc, ci, cj, ck);
              if (coef != 0.0 && ci == I && cj == J && ck == K)
                acc += coef * double(C.b[cidx(gc, I + di, J + dj, K + dk)]);
            }
        if (acc != 0.0) {
          const long long id = cidx(gc, I, J, K);
          C.b[id] = T(double(C.b[id]) + acc);
        }
      }
      __syncthreads();
    }
  }
  // coarsest level: sweeps from zero. With a single interior node (3 nodes a
  // side) the first sweep is already the fixed point (its neighbours are
  // boundary zeros), so the remaining sweeps, which would rewrite the same
  // value, are skipped.
  {
    const TailLevel<Coef, T>& L = lv[nlev - 1];
    const GridDev& g = L.g;
    const int total = (g.nx - 2) * (g.ny - 2) * (g.dim == 3 ? g.nz - 2 : 1);
    tail_zero(L);
    tail_sweeps(L, nlev == 1 ? rhs0 : L.b, total == 1 ? 1 : coarse_iters, 0);
  }
  // up: prolong-add, post-smooth
  for (int l = nlev - 2; l >= 0; --l) {
    const TailLevel<Coef, T>& F = lv[l];
    const TailLevel<Coef, T>& C = lv[l + 1];
    const GridDev& gf = F.g;
    const GridDev& gc = C.g;
    const int xmode = map_mode(gf.nx, gc.nx), ymode = map_mode(gf.ny, gc.ny);
    const int zmode = gf.dim == 3 ? map_mode(gf.nz, gc.nz) : 0;
    const int total = (gf.nx - 2) * (gf.ny - 2) * (gf.dim == 3 ? gf.nz - 2 : 1);
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int i, j, k;
      tail_decode<Coef, T>(gf, t, i, j, k);
      int I0, J0, K0 = 0;
      double tx, ty, tz = 0.0;
      coarse_pos(i, gf.nx, gc.nx, xmode, I0, tx);
      coarse_pos(j, gf.ny, gc.ny, ymode, J0, ty);
      if (gf.dim == 3) coarse_pos(k, gf.nz, gc.nz, zmode, K0, tz);
      const int I1 = tx != 0.0 ? I0 + 1 : I0, J1 = ty != 0.0 ? J0 + 1 : J0;
      const int K1 = tz != 0.0 ? K0 + 1 : K0;
      const double c000 = ext_value(gc, C.x, I0, J0, K0), c100 = ext_value(gc, C.x, I1, J0, K0);
      const double c010 = ext_value(gc, C.x, I0, J1, K0), c110 = ext_value(gc, C.x, I1, J1, K0);
      const double c001 = ext_value(gc, C.x, I0, J0, K1), c101 = ext_value(gc, C.x, I1, J0, K1);
      const double c011 = ext_value(gc, C.x, I0, J1, K1), c111 = ext_value(gc, C.x, I1, J1, K1);
      const double x00 = (1.0 - tx) * c000 + tx * c100, x10 = (1.0 - tx) * c010 + tx * c110;
      const double x01 = (1.0 - tx) * c001 + tx * c101, x11 = (1.0 - tx) * c011 + tx * c111;
      const double y0 = (1.0 - ty) * x00 + ty * x10, y1 = (1.0 - ty) * x01 + ty * x11;
      const double v = (1.0 - tz) * y0 + tz * y1;
      const long long id = ((long long)k * gf.ny + j) * gf.nx + i;
      F.x[id] = T(double(F.x[id]) + v);
    }
    __syncthreads();
    tail_sweeps(F, l == 0 ? rhs0 : F.b, post, 1);
  }
}

}  // namespace pdeb
