// Whole red-black Gauss-Seidel sweep in one pass over HBM for the large 3D
// levels of the MG hierarchy (k_rbgs_march).
//
// Two colour passes (k_rbgs) each read all of x and k and half-use every
// 32-byte sector of b and of the written x, about 31 B of DRAM traffic per
// node per pass. One sweep needs only x read and written once and k and b
// read once: 32 B per node. This kernel gets there by marching each block
// through z over a 64 x 8 tile of interior (i, j) columns:
//
//   step p:  first colour on plane p over the tile plus a one-node ring
//            (66 x 10), from old values, in place in the staged plane;
//            one barrier;
//            second colour on plane p-1 over the tile, from the new
//            first-colour values of planes p-2 .. p; both colours of plane
//            p-1 go to x_out.
//
// Old x and k are staged per plane over the tile plus a two-node ring
// (68 x 12), b over the one-node ring, in shared-memory rings of 6 / 6 / 5
// planes; the loads of plane p+3 are issued during step p into registers and
// stored to their slot during step p+1, so a full step of work covers their
// latency and each step needs a single barrier (the ring depths are the live
// planes of two consecutive steps plus the one being written). Rows are
// stored split by column parity (even columns, then odd), so the nodes of one
// colour in a row, and each of their neighbours, are consecutive words: warp
// accesses to shared memory are free of bank conflicts.
//
// The first-colour values on the ring are recomputed by every block from old
// values only, so blocks never read each other's results: the sweep reads
// x_in and writes x_out (distinct buffers) and is race free and
// deterministic. Each node update is the arithmetic of k_rbgs (the stencil of
// CoefConst / CoefDivk in the same order, fold_faces, nb_sum, one IEEE
// division), so a sweep gives the two colour passes' values. zero_in: x_in is
// identically zero (the first sweep of a V-cycle level) and is not read.
// DOT: the sum over the updated nodes of b * (new x) is reduced over the grid
// and handed to `post` (the last sweep of the finest level gives r.z of
// preconditioned CG, since b is r there).
#pragma once

#include "kernels.cuh"

namespace pdeb {

constexpr int kMTx = 64, kMTy = 8;                  // tile of interior columns
constexpr int kMX2 = kMTx + 4, kMY2 = kMTy + 4;     // staged x, k: 68 x 12
constexpr int kMX1 = kMTx + 2, kMY1 = kMTy + 2;     // staged b, first colour: 66 x 10
constexpr int kMH2 = kMX2 / 2, kMH1 = kMX1 / 2;     // half rows: 34, 33
constexpr int kMN2 = kMX2 * kMY2, kMN1 = kMX1 * kMY1;  // 816, 660
constexpr int kMXSlots = 6, kMKSlots = 6, kMBSlots = 5;
constexpr int kMThreads = 256;
constexpr int kMLd2 = (kMN2 + kMThreads - 1) / kMThreads;  // 4 staged x/k cells per thread
constexpr int kMLd1 = (kMN1 + kMThreads - 1) / kMThreads;  // 3 staged b cells per thread
constexpr int kMRed = kMH1 * kMY1;                         // 330 first-colour cells per plane
static_assert(kMTx == 2 * 32 && kMTy * 32 == kMThreads, "one warp per tile row, two columns per lane");

template <class Coef>
struct MarchK {
  static constexpr bool kHasK = false;
  __device__ static const double* field(const Coef&) { return nullptr; }
};
template <>
struct MarchK<CoefDivk<double>> {
  static constexpr bool kHasK = true;
  __device__ static const double* field(const CoefDivk<double>& c) { return c.k; }
};

template <class Coef>
constexpr size_t march_smem_bytes() {
  return sizeof(double) * ((size_t)kMXSlots * kMN2 + (MarchK<Coef>::kHasK ? (size_t)kMKSlots * kMN2 : 0) +
                           (size_t)kMBSlots * kMN1);
}

// split-row index of staged cell (row r, column c)
__device__ __forceinline__ int ms2(int r, int c) { return r * kMX2 + (c & 1) * kMH2 + (c >> 1); }
__device__ __forceinline__ int ms1(int r, int c) { return r * kMX1 + (c & 1) * kMH1 + (c >> 1); }

template <class Coef, bool DOT = false, class Post = NoPost>
__global__ void __launch_bounds__(kMThreads, 2)
    k_rbgs_march(GridDev g, Coef cf, const double* __restrict__ b, const double* __restrict__ xin,
                 double* __restrict__ xout, int first, int zero_in, const Ctl* ctl, RedSlot slot = RedSlot{},
                 Post post = Post{}) {
  if (ctl_skip(ctl)) return;
  extern __shared__ double m_smem[];
  constexpr bool kK = MarchK<Coef>::kHasK;
  double* SX = m_smem;                                // [kMXSlots][kMN2]
  double* SK = SX + kMXSlots * kMN2;                  // [kMKSlots][kMN2] (divergence form only)
  double* SB = SK + (kK ? kMKSlots * kMN2 : 0);       // [kMBSlots][kMN1]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int X0 = 1 + blockIdx.x * kMTx, Y0 = 1 + blockIdx.y * kMTy;  // first interior column of the tile
  // interior planes [1, nz-1) split into gridDim.z chunks
  const int len = g.nz - 2;
  const int chunk = (len + gridDim.z - 1) / gridDim.z;
  const int k0 = 1 + blockIdx.z * chunk, k1 = min(g.nz - 1, k0 + chunk);
  const double* kfield = MarchK<Coef>::field(cf);
  const long long sxy = g.sxy;
  double acc[1] = {0.0};

  // x-y offsets of this thread's staged cells (fixed for every plane), -1 off the grid
  long long o2[kMLd2], o1[kMLd1];
  int s2[kMLd2], s1[kMLd1];
#pragma unroll
  for (int u = 0; u < kMLd2; ++u) {
    const int t = tid + u * kMThreads;
    const int r = t / kMX2, c = t % kMX2;
    const int gi = X0 - 2 + c, gj = Y0 - 2 + r;
    o2[u] = (t < kMN2 && gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny) ? (long long)gj * g.nx + gi : -1;
    s2[u] = t < kMN2 ? ms2(r, c) : -1;
  }
#pragma unroll
  for (int u = 0; u < kMLd1; ++u) {
    const int t = tid + u * kMThreads;
    const int r = t / kMX1, c = t % kMX1;
    const int gi = X0 - 1 + c, gj = Y0 - 1 + r;
    o1[u] = (t < kMN1 && gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny) ? (long long)gj * g.nx + gi : -1;
    s1[u] = t < kMN1 ? ms1(r, c) : -1;
  }

  // plane q of x (unless zero_in), k and b into registers (0 off the grid)
  double rx[kMLd2], rk[kMLd2], rb[kMLd1];
  auto fetch = [&](int q) {
    const bool qin = q >= 0 && q < g.nz;
    const long long base = (long long)q * sxy;
#pragma unroll
    for (int u = 0; u < kMLd2; ++u) {
      const bool in = qin && o2[u] >= 0;
      rx[u] = (in && !zero_in) ? __ldg(xin + base + o2[u]) : 0.0;
      if constexpr (kK) rk[u] = in ? __ldg(kfield + base + o2[u]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kMLd1; ++u) rb[u] = (qin && o1[u] >= 0) ? __ldg(b + base + o1[u]) : 0.0;
  };
  auto xslot = [&](int q) { return SX + ((q + 2 * kMXSlots) % kMXSlots) * kMN2; };
  auto kslot = [&](int q) { return SK + ((q + 2 * kMKSlots) % kMKSlots) * kMN2; };
  auto bslot = [&](int q) { return SB + ((q + 2 * kMBSlots) % kMBSlots) * kMN1; };
  auto store = [&](int q) {
    double* sx = xslot(q);
    double* sk = kslot(q);
    double* sb = bslot(q);
#pragma unroll
    for (int u = 0; u < kMLd2; ++u)
      if (s2[u] >= 0) {
        sx[s2[u]] = rx[u];
        if constexpr (kK) sk[s2[u]] = rk[u];
      }
#pragma unroll
    for (int u = 0; u < kMLd1; ++u)
      if (s1[u] >= 0) sb[s1[u]] = rb[u];
  };

  // Gauss-Seidel value at staged cell (r, c) of plane p (global gi, gj) from
  // the centre, lower and upper planes of x and k
  auto update = [&](int r, int c, int gi, int gj, int p, const double* xc, const double* xm, const double* xp,
                    const double* kcp, const double* kmp, const double* kpp, double bv) -> double {
    const int q = ms2(r, c), qxm = ms2(r, c - 1), qxp = ms2(r, c + 1), qym = ms2(r - 1, c), qyp = ms2(r + 1, c);
    Stencil<double> s;
    if constexpr (kK) {
      // the expressions of CoefDivk::at, in its order
      const double kc = kcp[q];
      const double kxm = 0.5 * (kc + kcp[qxm]), kxp = 0.5 * (kc + kcp[qxp]);
      const double kym = 0.5 * (kc + kcp[qym]), kyp = 0.5 * (kc + kcp[qyp]);
      s.xm = -kxm * cf.ihx2 - cf.cx;
      s.xp = -kxp * cf.ihx2 + cf.cx;
      s.ym = -kym * cf.ihy2 - cf.dyc;
      s.yp = -kyp * cf.ihy2 + cf.dyc;
      double cc = (kxm + kxp) * cf.ihx2 + (kym + kyp) * cf.ihy2;
      const double kzm = 0.5 * (kc + kmp[q]), kzp = 0.5 * (kc + kpp[q]);
      s.zm = -kzm * cf.ihz2 - cf.dzc;
      s.zp = -kzp * cf.ihz2 + cf.dzc;
      cc += (kzm + kzp) * cf.ihz2;
      s.c = cc + cf.e;
    } else {
      s = cf.template at<double>(g, 0);
    }
    if (gi == 1 || gi == g.nx - 2 || gj == 1 || gj == g.ny - 2 || p == 1 || p == g.nz - 2)
      fold_faces<double>(g, gi, gj, p, s, nullptr);
    return (bv - nb_sum<double>(s, xc[qxp], xc[qxm], xc[qyp], xc[qym], xp[q], xm[q], 3)) / s.c;
  };

  // first colour on plane p over the tile plus its ring, in place in slot p
  auto first_plane = [&](int p) {
    if (p < 1 || p > g.nz - 2) return;  // boundary planes keep x_in's (zero) values
    double* xc = xslot(p);
    const double* xm = xslot(p - 1);
    const double* xp = xslot(p + 1);
    const double* kc = kslot(p);
    const double* km = kslot(p - 1);
    const double* kp = kslot(p + 1);
    const double* bb = bslot(p);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = tid + u * kMThreads;
      if (t >= kMRed) break;
      const int r1 = t / kMH1, kk = t % kMH1;           // ring row, k-th first-colour cell of the row
      const int gj = Y0 - 1 + r1;
      const int par = (X0 - 1 + gj + p + first) & 1;    // column 0 of the ring row is first colour iff par == 0
      const int c1 = 2 * kk + par;                       // ring column
      const int gi = X0 - 1 + c1;
      if (gi < 1 || gi > g.nx - 2 || gj < 1 || gj > g.ny - 2) continue;
      xc[ms2(r1 + 1, c1 + 1)] =
          update(r1 + 1, c1 + 1, gi, gj, p, xc, xm, xp, kc, km, kp, bb[ms1(r1, c1)]);
    }
  };

  // second colour on plane p over the tile; both colours of plane p to x_out
  auto second_plane = [&](int p) {
    const int gj = Y0 + warp;
    const double* xc = xslot(p);
    const double* xm = xslot(p - 1);
    const double* xp = xslot(p + 1);
    const double* kc = kslot(p);
    const double* km = kslot(p - 1);
    const double* kp = kslot(p + 1);
    const double* bb = bslot(p);
    const int d1 = (X0 + gj + p + first) & 1;  // column offset of the first-colour node of the lane's pair
    const int gi1 = X0 + 2 * lane + d1, gi2 = X0 + 2 * lane + (d1 ^ 1);
    if (gj > g.ny - 2) return;
    const long long row = (long long)p * sxy + (long long)gj * g.nx;
    if (gi2 <= g.nx - 2) {
      const int c2 = gi2 - X0 + 2;
      const double bv = bb[ms1(warp + 1, c2 - 1)];
      const double v = update(warp + 2, c2, gi2, gj, p, xc, xm, xp, kc, km, kp, bv);
      xout[row + gi2] = v;
      if constexpr (DOT) acc[0] += bv * v;
    }
    if (gi1 <= g.nx - 2) {
      const int c1 = gi1 - X0 + 2;
      const double v = xc[ms2(warp + 2, c1)];
      xout[row + gi1] = v;
      if constexpr (DOT) acc[0] += bb[ms1(warp + 1, c1 - 1)] * v;
    }
  };

  if (k0 < k1) {
    // planes k0-2 .. k0 staged, k0+1 in flight
    for (int q = k0 - 2; q <= k0; ++q) {
      fetch(q);
      store(q);
    }
    fetch(k0 + 1);
    __syncthreads();
    for (int p = k0 - 1; p <= k1; ++p) {
      first_plane(p);
      if (p + 2 <= k1 + 1) store(p + 2);   // plane p+2 (fetched during the previous step)
      if (p + 3 <= k1 + 1) fetch(p + 3);   // in flight during the rest of this step and the next
      __syncthreads();
      if (p - 1 >= k0) second_plane(p - 1);
    }
  }
  if constexpr (DOT) grid_reduce<1, false>(acc, slot, post);
}

}  // namespace pdeb
