// Whole red-black Gauss-Seidel sweep in one pass over HBM for the large 3D
// levels of the MG hierarchy (k_rbgs_march).
//
// Two colour passes (k_rbgs) each read all of x and k and half-use every
// 32-byte sector of b and of the written x, about 31 B of DRAM traffic per
// node per pass. One sweep needs only x read and written once and k and b
// read once: 32 B per node. This kernel gets there by marching each block
// through z over a 64 x 8 tile of interior (i, j) columns:
//
//   step p:  A  first colour on plane p over the tile (warps 0-7, one tile
//               row each), from old values, in place in the staged plane;
//            one barrier;
//            B  second colour on plane p-1 over the tile from the new
//               first-colour values of planes p-2 .. p, both colours of
//               plane p-1 to x_out (warps 0-7); meanwhile warps 8-10 update
//               the first colour of plane p on the one-node ring around the
//               tile, which the second colour of plane p reads in step p+1.
//
// Every thread updates at most one node per phase, so a step costs two
// updates on the critical path.
// Old x and k are staged per plane over the tile plus a two-node ring
// (68 x 12) in shared-memory rings of 8 planes by asynchronous copies
// (cp.async, zero-filled off the grid): the copies of plane p+4 are issued in
// step p and waited for in step p+2, so three planes are always in flight and
// each step needs a single barrier (the ring holds the 5 planes that two
// consecutive steps read plus the 3 in flight). b is read once per node into
// registers, three steps before its use. Rows are stored split by column parity (even columns, then odd),
// so the nodes of one colour in a row, and each of their neighbours, are
// consecutive words: warp accesses to shared memory are free of bank
// conflicts.
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
constexpr int kMX1 = kMTx + 2;                      // one-node ring around the tile: 66 wide
constexpr int kMH2 = kMX2 / 2, kMH1 = kMX1 / 2;     // half rows: 34, 33
constexpr int kMN2 = kMX2 * kMY2;                   // 816 staged cells per plane
constexpr int kMSlots = 8;                           // x and k planes: 5 live + 3 in flight
constexpr int kMRowWarps = kMTy;                    // warps 0..7: one tile row each, two columns per lane
constexpr int kMRing = kMH1 * 2 + (kMTy * 2) / 2;   // first-colour cells of the ring: 33 + 33 + 8 = 74
constexpr int kMRingWarps = (kMRing + 31) / 32;     // warps 8..10
constexpr int kMThreads = 32 * (kMRowWarps + kMRingWarps);  // 352
constexpr int kMLd2 = (kMN2 + kMThreads - 1) / kMThreads;  // 3 staged x/k cells per thread
static_assert(kMTx == 2 * 32, "two tile columns per lane");

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
  return sizeof(double) * (size_t)kMSlots * kMN2 * (MarchK<Coef>::kHasK ? 2 : 1);
}

// 8-byte asynchronous global -> shared copy; src_bytes 0 zero-fills the word
__device__ __forceinline__ void m_cp8(double* smem, const double* gmem, int src_bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void m_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// all but the two most recent groups of this thread's copies have landed
__device__ __forceinline__ void m_wait_all_but_two() { asm volatile("cp.async.wait_group 2;\n" ::: "memory"); }

// split-row index of staged cell (row r, column c)
__host__ __device__ __forceinline__ int ms2(int r, int c) { return r * kMX2 + (c & 1) * kMH2 + (c >> 1); }

// One node's place in the staged planes for one plane parity: split index q,
// the offsets of its x neighbours (a column of the other parity sits in the
// other half-row), grid position and whether it is interior / face-adjacent
// in x-y.
struct MCell {
  int q, oxp, oxm, gi, gj;
  long long go;  // gj * nx + gi: offset of the node in its plane
  bool in, near;
};

__device__ __forceinline__ MCell mcell(const GridDev& g, int X0, int Y0, int r, int c, bool valid) {
  MCell m;
  m.q = ms2(r, c);
  m.oxp = (c & 1) ? 1 - kMH2 : kMH2;       // column c+1
  m.oxm = (c & 1) ? -kMH2 : kMH2 - 1;      // column c-1
  m.gi = X0 - 2 + c;
  m.gj = Y0 - 2 + r;
  m.go = (long long)m.gj * g.nx + m.gi;
  m.in = valid && m.gi >= 1 && m.gi <= g.nx - 2 && m.gj >= 1 && m.gj <= g.ny - 2;
  m.near = m.gi == 1 || m.gi == g.nx - 2 || m.gj == 1 || m.gj == g.ny - 2;
  return m;
}

template <class Coef, bool DOT = false, class Post = NoPost>
__global__ void __launch_bounds__(kMThreads, 2)
    k_rbgs_march(GridDev g, Coef cf, const double* __restrict__ b, const double* __restrict__ xin,
                 double* __restrict__ xout, int first, int zero_in, const Ctl* ctl, RedSlot slot = RedSlot{},
                 Post post = Post{}) {
  if (ctl_skip(ctl)) return;
  extern __shared__ double m_smem[];
  constexpr bool kK = MarchK<Coef>::kHasK;
  double* SX = m_smem;               // [kMSlots][kMN2]
  double* SK = SX + kMSlots * kMN2;  // [kMSlots][kMN2] (divergence form only)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool row_warp = warp < kMRowWarps;
  const int X0 = 1 + blockIdx.x * kMTx, Y0 = 1 + blockIdx.y * kMTy;  // first interior column / row of the tile
  // interior planes [1, nz-1) split into gridDim.z chunks
  const int len = g.nz - 2;
  const int chunk = (len + gridDim.z - 1) / gridDim.z;
  const int k0 = 1 + blockIdx.z * chunk, k1 = min(g.nz - 1, k0 + chunk);
  const double* kfield = MarchK<Coef>::field(cf);
  const long long sxy = g.sxy;
  double acc[1] = {0.0};

  // The cells of this thread, per plane parity pi = p & 1. Row warps: the
  // first-colour node of the lane's column pair on plane p, which is also the
  // pair's second-colour node on plane p-1. Ring warps: the t-th first-colour
  // node of the ring on plane p (rows above and below the tile, then the
  // side columns).
  auto make_cell = [&](int pi) -> MCell {
    if (row_warp) {
      const int r = warp + 2;
      const int d = (X0 + Y0 + warp + pi + first) & 1;
      return mcell(g, X0, Y0, r, 2 + 2 * lane + d, true);
    }
    const int t = tid - 32 * kMRowWarps;
    int r, c;
    if (t < 2 * kMH1) {
      r = t < kMH1 ? 1 : kMY2 - 2;
      const int e = (X0 + Y0 - 2 + r + pi + first) & 1;  // parity of the row's first-colour columns
      c = 2 + 2 * (t % kMH1) - e;
    } else {
      r = 2 + (t - 2 * kMH1);
      const int e = (X0 + Y0 - 2 + r + pi + first) & 1;
      c = e ? 1 : kMX2 - 2;
    }
    return mcell(g, X0, Y0, r < kMY2 - 1 ? r : kMY2 - 2, c, t < kMRing);
  };
  // cells of the planes k0-1, k0+1, ... (ca) and k0, k0+2, ... (cb)
  const MCell ca = make_cell((k0 - 1) & 1), cb = make_cell(k0 & 1);

  // x-y offsets of this thread's staged cells (fixed for every plane), -1 off the grid
  long long o2[kMLd2];
  int s2[kMLd2];
#pragma unroll
  for (int u = 0; u < kMLd2; ++u) {
    const int t = tid + u * kMThreads;
    const int r = t / kMX2, c = t % kMX2;
    const int gi = X0 - 2 + c, gj = Y0 - 2 + r;
    o2[u] = (t < kMN2 && gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny) ? (long long)gj * g.nx + gi : -1;
    s2[u] = t < kMN2 ? ms2(r, c) : -1;
  }
  auto xslot = [&](int q) { return SX + ((q + 2 * kMSlots) % kMSlots) * kMN2; };
  auto kslot = [&](int q) { return SK + ((q + 2 * kMSlots) % kMSlots) * kMN2; };
  // asynchronous copies of plane q of x (zeros with zero_in) and k into their
  // slots, zero-filled off the grid, as one commit group
  auto stage = [&](int q) {
    const bool qin = q >= 0 && q < g.nz;
    const long long base = (long long)q * sxy;
    double* sx = xslot(q);
    double* sk = kslot(q);
#pragma unroll
    for (int u = 0; u < kMLd2; ++u) {
      if (s2[u] < 0) continue;
      const bool in = qin && o2[u] >= 0;
      m_cp8(sx + s2[u], in ? xin + base + o2[u] : xin, (in && !zero_in) ? 8 : 0);
      if constexpr (kK) m_cp8(sk + s2[u], in ? kfield + base + o2[u] : kfield, in ? 8 : 0);
    }
    m_commit();
  };

  // divergence-form face factors: (k_i + k_nb) * (1/(2 h^2)) equals the
  // CoefDivk expression 0.5 (k_i + k_nb) * 1/h^2 exactly (scaling by 2 is exact)
  double hx = 0.0, hy = 0.0, hz = 0.0;
  if constexpr (kK) {
    hx = 0.5 * cf.ihx2;
    hy = 0.5 * cf.ihy2;
    hz = 0.5 * cf.ihz2;
  }

  // Gauss-Seidel value of cell m on plane p from the staged planes around it
  auto update = [&](const MCell& m, int p, const double* xc, const double* xm, const double* xp, double bv) -> double {
    const int q = m.q;
    Stencil<double> s;
    if constexpr (kK) {
      const double* kc = kslot(p);
      const double k0v = kc[q];
      const double sxm = k0v + kc[q + m.oxm], sxp = k0v + kc[q + m.oxp];
      const double sym = k0v + kc[q - kMX2], syp = k0v + kc[q + kMX2];
      const double szm = k0v + kslot(p - 1)[q], szp = k0v + kslot(p + 1)[q];
      s.xm = -sxm * hx - cf.cx;
      s.xp = -sxp * hx + cf.cx;
      s.ym = -sym * hy - cf.dyc;
      s.yp = -syp * hy + cf.dyc;
      double cc = (sxm + sxp) * hx + (sym + syp) * hy;
      s.zm = -szm * hz - cf.dzc;
      s.zp = -szp * hz + cf.dzc;
      cc += (szm + szp) * hz;
      s.c = cc + cf.e;
    } else {
      s = cf.template at<double>(g, 0);
    }
    if (m.near || p == 1 || p == g.nz - 2) fold_faces<double>(g, m.gi, m.gj, p, s, nullptr);
    return (bv - nb_sum<double>(s, xc[q + m.oxp], xc[q + m.oxm], xc[q + kMX2], xc[q - kMX2], xp[q], xm[q], 3)) /
           s.c;
  };

  // first colour of plane p at this thread's cell, in place in slot p
  auto first_cell = [&](const MCell& m, int p, double bv) {
    double* xc = xslot(p);
    xc[m.q] = update(m, p, xc, xslot(p - 1), xslot(p + 1), bv);
  };
  // b of plane q at this thread's cells ca and cb (0 off the interior), into
  // registers three steps before use
  auto load_b = [&](int q, double (&dst)[2]) {
    const bool qin = q >= 1 && q <= g.nz - 2;
    const long long base = (long long)q * sxy;
    dst[0] = (qin && ca.in) ? __ldg(b + base + ca.go) : 0.0;
    dst[1] = (qin && cb.in) ? __ldg(b + base + cb.go) : 0.0;
  };

  if (k0 < k1) {
    // planes k0-2 .. k0 landed, k0+1 and k0+2 in flight
    for (int q = k0 - 2; q <= k0 + 2; ++q) stage(q);
    m_wait_all_but_two();
    // b of planes k0-1 .. k0+1; B3 gets plane k0+2 at the end of the first step
    double B0[2], B1[2], B2[2], B3[2] = {0.0, 0.0};
    load_b(k0 - 1, B0);
    load_b(k0, B1);
    load_b(k0 + 1, B2);
    __syncthreads();
    // one step; cm: this thread's cell on plane p (register index im of the
    // b pairs), co: on planes p-1 and p+1; bprev / bcur: b of planes p-1 / p,
    // bprev reloaded with plane p+3 at the end
    auto step = [&](int p, const MCell& cm, const MCell& co, int im, double (&bprev)[2], double (&bcur)[2]) {
      const bool plane_in = p >= 1 && p <= g.nz - 2;
      // A: first colour of plane p on the tile (read by the second colour of
      // plane p-1 below, across the barrier)
      if (row_warp && plane_in && cm.in) first_cell(cm, p, im ? bcur[1] : bcur[0]);
      // plane p+4 in flight during the next three steps; plane p+2 (issued
      // two steps ago) landed, and visible after the barrier
      if (p + 4 <= k1 + 1)
        stage(p + 4);
      else
        m_commit();  // an empty group keeps the wait below uniform
      m_wait_all_but_two();
      __syncthreads();
      if (row_warp) {
        // B: second colour of plane p-1 (same column as the first colour of
        // plane p) and both colours of plane p-1 to x_out
        const int q = p - 1;
        if (q >= k0) {
          const MCell& m = cm;
          const MCell& f = co;
          const double* xc = xslot(q);
          const long long base = (long long)q * sxy;
          if (m.in) {
            const double bv = im ? bprev[1] : bprev[0];
            const double v = update(m, q, xc, xslot(q - 1), xslot(p), bv);
            xout[base + m.go] = v;
            if constexpr (DOT) acc[0] += bv * v;
          }
          if (f.in) {
            const double v = xc[f.q];
            xout[base + f.go] = v;
            if constexpr (DOT) acc[0] += (im ? bprev[0] : bprev[1]) * v;
          }
        }
      } else if (plane_in && p >= k0 && p < k1 && cm.in) {
        // B: first colour of plane p on the ring (read by the second colour
        // of plane p in the next step, across its barrier)
        first_cell(cm, p, im ? bcur[1] : bcur[0]);
      }
      load_b(p + 3, bprev);
    };
    // unrolled by four so every b register pair has a fixed name
    for (int p = k0 - 1; p <= k1; p += 4) {
      step(p, ca, cb, 0, B3, B0);
      if (p + 1 <= k1) step(p + 1, cb, ca, 1, B0, B1);
      if (p + 2 <= k1) step(p + 2, ca, cb, 0, B1, B2);
      if (p + 3 <= k1) step(p + 3, cb, ca, 1, B2, B3);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  if constexpr (DOT) grid_reduce<1, false>(acc, slot, post);
}

}  // namespace pdeb
