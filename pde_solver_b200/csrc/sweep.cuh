// Single-pass red-black Gauss-Seidel sweep with shared-memory staging.
//
// A block owns a 32 x 8 tile of (i, j) columns (global x in [X0, X0+32),
// y in [Y0, Y0+8)) and a chunk of planes [k0, k1). It marches in z: at step p
// it updates the first colour on plane p over the tile plus a one-node ring
// (R1, 34 x 10) from the old field, then the second colour on plane p-1 over
// the tile from the new first-colour values. Old x, k and b of each plane are
// staged once in shared memory over the tile plus a two-node ring (R2,
// 36 x 12; b over R1) with cp.async, one plane ahead of use, so every array is
// read from HBM once per sweep (the ring re-reads hit L2) instead of once per
// colour pass. The first-colour values on the ring are recomputed by each
// block from old values only, so the sweep is race free; it reads x_in and
// writes x_out (distinct buffers). Every node update is the arithmetic of
// k_rbgs (same stencil, same neighbour values), so the result equals two
// colour passes up to rounding. zero_in: x_in is identically zero (first
// sweep of a V-cycle level) and is not read.
#pragma once

#include "kernels.cuh"

namespace pdeb {

constexpr int kSwX = 32, kSwY = 8;                 // tile
constexpr int kR1X = kSwX + 2, kR1Y = kSwY + 2;     // first-colour ring
constexpr int kR2X = kSwX + 4, kR2Y = kSwY + 4;     // staged old x / k
constexpr int kR1N = kR1X * kR1Y, kR2N = kR2X * kR2Y;
constexpr int kSwXSlots = 4, kSwKSlots = 5, kSwBSlots = 4, kSwRSlots = 3;
constexpr int kSwThreads = kSwX * kSwY;
constexpr size_t kSwSmemBytes =
    sizeof(double) * ((size_t)kSwXSlots * kR2N + (size_t)kSwKSlots * kR2N + (size_t)kSwBSlots * kR1N +
                      (size_t)kSwRSlots * kR1N);

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid ? 8 : 0;  // 0: the shared word is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <class Coef>
struct SweepK {
  static constexpr bool kHasK = false;
  __device__ static const double* field(const Coef&) { return nullptr; }
};
template <>
struct SweepK<CoefDivk<double>> {
  static constexpr bool kHasK = true;
  __device__ static const double* field(const CoefDivk<double>& c) { return c.k; }
};

// Stencil of the node at R2 position (a, b) of the staged planes: constant
// coefficients directly, divergence form from the staged k (the expressions of
// CoefDivk::at, in its order).
template <class Coef>
__device__ __forceinline__ Stencil<double> sweep_stencil(const GridDev& g, const Coef& cf, const double* kc,
                                                         const double* km, const double* kp, int a, int b,
                                                         long long id) {
  if constexpr (SweepK<Coef>::kHasK) {
    const int q = b * kR2X + a;
    const double k0 = kc[q];
    const double kxm = 0.5 * (k0 + kc[q - 1]), kxp = 0.5 * (k0 + kc[q + 1]);
    const double kym = 0.5 * (k0 + kc[q - kR2X]), kyp = 0.5 * (k0 + kc[q + kR2X]);
    Stencil<double> s;
    s.xm = -kxm * cf.ihx2 - cf.cx;
    s.xp = -kxp * cf.ihx2 + cf.cx;
    s.ym = -kym * cf.ihy2 - cf.dyc;
    s.yp = -kyp * cf.ihy2 + cf.dyc;
    double c = (kxm + kxp) * cf.ihx2 + (kym + kyp) * cf.ihy2;
    if (g.dim == 3) {
      const double kzm = 0.5 * (k0 + km[q]), kzp = 0.5 * (k0 + kp[q]);
      s.zm = -kzm * cf.ihz2 - cf.dzc;
      s.zp = -kzp * cf.ihz2 + cf.dzc;
      c += (kzm + kzp) * cf.ihz2;
    } else {
      s.zm = s.zp = 0.0;
    }
    s.c = c + cf.e;
    return s;
  } else {
    return cf.template at<double>(g, id);
  }
}

template <class Coef>
__global__ void __launch_bounds__(kSwThreads) k_rbgs_sweep(GridDev g, Coef cf, const double* __restrict__ b,
                                                           const double* __restrict__ xin,
                                                           double* __restrict__ xout, int first, int zero_in,
                                                           const Ctl* ctl) {
  if (ctl_skip(ctl)) return;
  extern __shared__ double sw_smem[];
  double* SX = sw_smem;                       // [kSwXSlots][kR2N]
  double* SK = SX + kSwXSlots * kR2N;         // [kSwKSlots][kR2N]
  double* SB = SK + kSwKSlots * kR2N;         // [kSwBSlots][kR1N]
  double* SR = SB + kSwBSlots * kR1N;         // [kSwRSlots][kR1N]
  const int tid = threadIdx.x;
  const int X0 = blockIdx.x * kSwX, Y0 = blockIdx.y * kSwY;
  const bool is3 = g.dim == 3;
  const int kb = is3 ? 1 : 0, ke = is3 ? g.nz - 1 : 1;  // interior planes
  const int len = ke - kb;
  const int chunk = (len + gridDim.z - 1) / gridDim.z;
  const int k0 = kb + blockIdx.z * chunk, k1 = min(ke, k0 + chunk);
  if (k0 >= k1) return;
  const double* kfield = SweepK<Coef>::field(cf);
  const long long sxy = g.sxy;

  // ---- per-thread positions, fixed for every plane
  // staged R2 cells t = tid, tid + blockDim (x and k) and R1 cells (b): global x-y
  // offset, or -1 outside the grid
  long long l2[2], l1[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int t2 = tid + u * kSwThreads;
    const int gi = X0 - 2 + t2 % kR2X, gj = Y0 - 2 + t2 / kR2X;
    l2[u] = (t2 < kR2N && gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny) ? (long long)gj * g.nx + gi : -1;
    const int t1 = tid + u * kSwThreads;
    const int hi = X0 - 1 + t1 % kR1X, hj = Y0 - 1 + t1 / kR1X;
    l1[u] = (t1 < kR1N && hi >= 0 && hi < g.nx && hj >= 0 && hj < g.ny) ? (long long)hj * g.nx + hi : -1;
  }
  // Colour-compacted cells: at plane p thread t < 170 updates the t-th
  // first-colour cell of R1 (17 per row of 34) and thread t < 128 the t-th
  // second-colour cell of the tile (16 per row of 32); the column within the
  // row follows the plane's parity, so active warps run full.
  constexpr int kRedPerRow = kR1X / 2, kRedCells = kR1N / 2;
  constexpr int kBlkPerRow = kSwX / 2, kBlkCells = kSwX * kSwY / 2;
  const int red_rb = tid / kRedPerRow, red_c = tid % kRedPerRow;
  const int red_gj = Y0 - 1 + red_rb;
  const int red_par = (first + X0 + 1 + red_gj) & 1;  // + p: parity of ra
  const int blk_tb = tid / kBlkPerRow, blk_c = tid % kBlkPerRow;
  const int blk_gj = Y0 + blk_tb;
  const int blk_par = (1 + first + X0 + blk_gj) & 1;  // + p: parity of ta
  struct Cell {
    int gi, gj, q, r;
  };

  // stage plane q (zero-filled outside the grid)
  auto load_plane = [&](int q, int sx_slot, int sk_slot, int sb_slot) {
    const bool qin = q >= 0 && q < g.nz;
    double* sx = SX + sx_slot * kR2N;
    double* sk = SK + sk_slot * kR2N;
    double* sb = SB + sb_slot * kR1N;
    const long long base = (long long)q * sxy;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t2 = tid + u * kSwThreads;
      if (t2 < kR2N) {
        const bool in = qin && l2[u] >= 0;
        const long long id = in ? base + l2[u] : 0;
        if (zero_in)
          sx[t2] = 0.0;
        else
          cp_async8(sx + t2, xin + id, in);
        if constexpr (SweepK<Coef>::kHasK) cp_async8(sk + t2, kfield + id, in);
      }
      const int t1 = tid + u * kSwThreads;
      if (t1 < kR1N) {
        const bool in = qin && l1[u] >= 0;
        cp_async8(sb + t1, b + (in ? base + l1[u] : 0), in);
      }
    }
    cp_async_commit();
  };

  // one Gauss-Seidel update of cell c on plane p from neighbour values nb
  // (stride nbx between rows), given the staged k and b
  auto update = [&](const Cell& c, int p, const double* kc, const double* km, const double* kp, double bv,
                    const double* nb, int ni, int nbx, const double* nbm, const double* nbp) -> double {
    const long long id = (long long)p * sxy + (long long)c.gj * g.nx + c.gi;
    Stencil<double> s = sweep_stencil<Coef>(g, cf, kc, km, kp, c.q % kR2X, c.q / kR2X, id);
    if (c.gi == 1 || c.gi == g.nx - 2 || c.gj == 1 || c.gj == g.ny - 2 || (is3 && (p == 1 || p == g.nz - 2)))
      fold_faces<double>(g, c.gi, c.gj, p, s, nullptr);
    const double zp = is3 ? nbp[ni] : 0.0;
    const double zm = is3 ? nbm[ni] : 0.0;
    return (bv - nb_sum<double>(s, nb[ni + 1], nb[ni - 1], nb[ni + nbx], nb[ni - nbx], zp, zm, g.dim)) / s.c;
  };

  // ring slots of plane p: x mod 4, k mod 5, b mod 4, red mod 3 (p >= -3)
  auto sx_of = [](int p) { return (p + 4) & 3; };
  auto sk_of = [](int p) { return (p + 5) % 5; };
  auto sb_of = [](int p) { return (p + 4) & 3; };
  auto sr_of = [](int p) { return (p + 3) % 3; };

  auto first_plane = [&](int p) {
    if (tid >= kRedCells) return;
    const double* xc = SX + sx_of(p) * kR2N;
    const double* xm = SX + sx_of(p - 1) * kR2N;
    const double* xp = SX + sx_of(p + 1) * kR2N;
    const double* kc = SK + sk_of(p) * kR2N;
    const double* km = SK + sk_of(p - 1) * kR2N;
    const double* kp = SK + sk_of(p + 1) * kR2N;
    const double* bb = SB + sb_of(p) * kR1N;
    double* rr = SR + sr_of(p) * kR1N;
    const int ra = 2 * red_c + ((red_par + p) & 1);
    Cell c{X0 - 1 + ra, red_gj, (red_rb + 1) * kR2X + ra + 1, red_rb * kR1X + ra};
    double v = 0.0;
    if (p >= kb && p < ke && c.gi >= 1 && c.gi <= g.nx - 2 && c.gj >= 1 && c.gj <= g.ny - 2) {
      v = update(c, p, kc, km, kp, bb[c.r], xc, c.q, kR2X, xm, xp);
      if (ra >= 1 && ra <= kSwX && red_rb >= 1 && red_rb <= kSwY && p >= k0 && p < k1)
        xout[(long long)p * sxy + (long long)c.gj * g.nx + c.gi] = v;
    }
    rr[c.r] = v;
  };

  auto second_plane = [&](int p) {
    if (tid >= kBlkCells) return;
    const int ta = 2 * blk_c + ((blk_par + p) & 1);
    Cell c{X0 + ta, blk_gj, (blk_tb + 2) * kR2X + ta + 2, (blk_tb + 1) * kR1X + ta + 1};
    if (!(c.gi >= 1 && c.gi <= g.nx - 2 && c.gj >= 1 && c.gj <= g.ny - 2)) return;
    const double* rc = SR + sr_of(p) * kR1N;
    const double* rm = SR + sr_of(p - 1) * kR1N;
    const double* rp = SR + sr_of(p + 1) * kR1N;
    const double* kc = SK + sk_of(p) * kR2N;
    const double* km = SK + sk_of(p - 1) * kR2N;
    const double* kp = SK + sk_of(p + 1) * kR2N;
    const double* bb = SB + sb_of(p) * kR1N;
    xout[(long long)p * sxy + (long long)c.gj * g.nx + c.gi] = update(c, p, kc, km, kp, bb[c.r], rc, c.r, kR1X, rm, rp);
  };

  if (!is3) {
    load_plane(0, 0, 0, 0);
    cp_async_wait_all();
    __syncthreads();
    first_plane(0);
    __syncthreads();
    second_plane(0);
    return;
  }
  // planes k0-2 .. k0 before the first step (p = k0 - 1)
  for (int q = k0 - 2; q <= k0; ++q) load_plane(q, sx_of(q), sk_of(q), sb_of(q));
  for (int p = k0 - 1; p <= k1; ++p) {
    cp_async_wait_all();
    __syncthreads();
    if (p + 2 <= k1 + 1) load_plane(p + 2, sx_of(p + 2), sk_of(p + 2), sb_of(p + 2));  // overlaps the updates
    first_plane(p);
    __syncthreads();
    if (p - 1 >= k0) second_plane(p - 1);
  }
  cp_async_wait_all();
}

}  // namespace pdeb
