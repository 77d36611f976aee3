// Device-side descriptors and inline stencil math shared by every kernel of
// libpdeb200. Layout: node-centred grid, flat index (k*ny + j)*nx + i with x
// fastest, identical to the reference (src/backends/cpu/cpu_utils.h:13-19), so
// fields cross the ABI without repacking.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pdeb {

enum Face { kLeft = 0, kRight, kBottom, kTop, kFront, kBack };
enum BcKind { kDirichlet = 0, kNeumann = 1, kRobin = 2 };
enum CoefKind { kConst = 0, kDivk = 1, kNodal = 2 };

// A face parameter is a scalar or a per-face-node array (face-local index:
// left/right j + ny*k, bottom/top i + nx*k, front/back i + nx*j).
struct FaceParam {
  double s;
  const double* a;
  __device__ __forceinline__ double at(int loc) const { return a ? a[loc] : s; }
};

struct FaceDev {
  int kind;
  int active;      // the face exists (x/y faces always, z faces in 3D)
  double h;        // spacing normal to the face
  FaceParam val, alpha, beta, gamma;  // reference closure inputs
  FaceParam c0, c1;                   // folded closure u_b = c0 + c1 * u_nb
};

struct GridDev {
  int nx, ny, nz, dim;
  long long n, sxy;
  FaceDev face[6];
};

// Seven stencil weights of one interior node in the reference's naming:
// value = c*u + (xp*u[i+1] + xm*u[i-1] + yp*u[j+1] + ym*u[j-1]) (+ zp*u[k+1] + zm*u[k-1]).
template <typename T>
struct Stencil {
  T c, xm, xp, ym, yp, zm, zp;
};

// Constant coefficients, precomputed on the host with the reference's own
// expressions (src/backends/cpu/solver.cpp:723-729) so they are bit-identical.
// Prefetch of the 32-byte sector holding p into L2 (no register result).
__device__ __forceinline__ void pf_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

struct CoefConst {
  double c, xm, xp, ym, yp, zm, zp;
  template <typename T, int D = 0>
  __device__ __forceinline__ Stencil<T> at(const GridDev&, long long) const {
    return Stencil<T>{T(c), T(xm), T(xp), T(ym), T(yp), T(zm), T(zp)};
  }
  __device__ __forceinline__ void prefetch(long long) const {}
};

template <typename KT>
__device__ __forceinline__ double load_k(const KT* k, long long id);
template <>
__device__ __forceinline__ double load_k<double>(const double* k, long long id) { return __ldg(k + id); }
template <>
__device__ __forceinline__ double load_k<float>(const float* k, long long id) { return (double)__ldg(k + id); }
template <>
__device__ __forceinline__ double load_k<__nv_bfloat16>(const __nv_bfloat16* k, long long id) {
  return (double)__bfloat162float(k[id]);
}

// Divergence form -div(k grad u) + convection + e*u with k at nodes and
// face values k_f = (k_i + k_nb)/2; constant k is the reference stencil with
// a = b = az = -k.
template <typename KT>
struct CoefDivk {
  const KT* k;
  double ihx2, ihy2, ihz2;  // 1/h^2
  double cx, dyc, dzc, e;   // c/(2dx), d/(2dy), dz/(2dz), e
  __device__ __forceinline__ void prefetch(long long id) const { pf_l2(k + id); }
  // D: the grid dimension when the caller knows it at compile time, else 0
  template <typename T, int D = 0>
  __device__ __forceinline__ Stencil<T> at(const GridDev& g, long long id) const {
    const bool d3 = D ? D == 3 : g.dim == 3;
    if constexpr (sizeof(T) == 4) {
      // FP32 stencils (preconditioner levels of the precision form) in FP32
      const float kc = float(load_k(k, id));
      const float kxm = 0.5f * (kc + float(load_k(k, id - 1))), kxp = 0.5f * (kc + float(load_k(k, id + 1)));
      const float kym = 0.5f * (kc + float(load_k(k, id - g.nx))), kyp = 0.5f * (kc + float(load_k(k, id + g.nx)));
      const float fx = float(ihx2), fy = float(ihy2);
      Stencil<T> s;
      s.xm = T(-kxm * fx - float(cx));
      s.xp = T(-kxp * fx + float(cx));
      s.ym = T(-kym * fy - float(dyc));
      s.yp = T(-kyp * fy + float(dyc));
      float c = (kxm + kxp) * fx + (kym + kyp) * fy;
      if (d3) {
        const float fz = float(ihz2);
        const float kzm = 0.5f * (kc + float(load_k(k, id - g.sxy))), kzp = 0.5f * (kc + float(load_k(k, id + g.sxy)));
        s.zm = T(-kzm * fz - float(dzc));
        s.zp = T(-kzp * fz + float(dzc));
        c += (kzm + kzp) * fz;
      } else {
        s.zm = s.zp = T(0);
      }
      s.c = T(c + float(e));
      return s;
    }
    const double kc = load_k(k, id);
    const double kxm = 0.5 * (kc + load_k(k, id - 1)), kxp = 0.5 * (kc + load_k(k, id + 1));
    const double kym = 0.5 * (kc + load_k(k, id - g.nx)), kyp = 0.5 * (kc + load_k(k, id + g.nx));
    Stencil<T> s;
    s.xm = T(-kxm * ihx2 - cx);
    s.xp = T(-kxp * ihx2 + cx);
    s.ym = T(-kym * ihy2 - dyc);
    s.yp = T(-kyp * ihy2 + dyc);
    double c = (kxm + kxp) * ihx2 + (kym + kyp) * ihy2;
    if (d3) {
      const double kzm = 0.5 * (kc + load_k(k, id - g.sxy)), kzp = 0.5 * (kc + load_k(k, id + g.sxy));
      s.zm = T(-kzm * ihz2 - dzc);
      s.zp = T(-kzp * ihz2 + dzc);
      c += (kzm + kzp) * ihz2;
    } else {
      s.zm = s.zp = T(0);
    }
    s.c = T(c + e);
    return s;
  }
};

// Per-node a,b,az,c,d,dz,e arrays (array-major). Divisions are IEEE and in the
// reference's order (src/backends/cpu/solver.cpp:855-866) for bit parity.
struct CoefNodal {
  const double* nodal;
  long long n;
  double dx2, dy2, dz2, tdx, tdy, tdz;  // dx*dx, ..., 2*dx, ...
  __device__ __forceinline__ void prefetch(long long) const {}
  template <typename T, int D = 0>
  __device__ __forceinline__ Stencil<T> at(const GridDev& g, long long id) const {
    const bool d3 = D ? D == 3 : g.dim == 3;
    const double a = __ldg(nodal + id), b = __ldg(nodal + n + id);
    const double c = __ldg(nodal + 3 * n + id), d = __ldg(nodal + 4 * n + id), e = __ldg(nodal + 6 * n + id);
    const double ax = __ddiv_rn(a, dx2), by = __ddiv_rn(b, dy2);
    const double cx = __ddiv_rn(c, tdx), dyc = __ddiv_rn(d, tdy);
    Stencil<T> s;
    s.xp = T(__dadd_rn(ax, cx));
    s.xm = T(__dsub_rn(ax, cx));
    s.yp = T(__dadd_rn(by, dyc));
    s.ym = T(__dsub_rn(by, dyc));
    if (d3) {
      const double az = __ldg(nodal + 2 * n + id), dzv = __ldg(nodal + 5 * n + id);
      const double cz = __ddiv_rn(az, dz2), dzc = __ddiv_rn(dzv, tdz);
      s.zp = T(__dadd_rn(cz, dzc));
      s.zm = T(__dsub_rn(cz, dzc));
      s.c = T(__dadd_rn(__dsub_rn(__dsub_rn(__dmul_rn(-2.0, ax), __dmul_rn(2.0, by)), __dmul_rn(2.0, cz)), e));
    } else {
      s.zp = s.zm = T(0);
      s.c = T(__dadd_rn(__dsub_rn(__dmul_rn(-2.0, ax), __dmul_rn(2.0, by)), e));
    }
    return s;
  }
};

// Folding of the boundary closure of face-adjacent interior nodes:
// diag += w_face * c1, the face term is dropped, and (optionally) w_face*c0
// is accumulated for the right-hand side.
template <typename T, int D = 0>
__device__ __forceinline__ void fold_faces(const GridDev& g, int i, int j, int k, Stencil<T>& s,
                                           double* bshift) {
  const bool d3 = D ? D == 3 : g.dim == 3;
  double sh = 0.0;
  if (i == 1) {
    const FaceDev& f = g.face[kLeft];
    const int loc = j + g.ny * k;
    s.c += s.xm * T(f.c1.at(loc));
    sh += double(s.xm) * f.c0.at(loc);
    s.xm = T(0);
  }
  if (i == g.nx - 2) {
    const FaceDev& f = g.face[kRight];
    const int loc = j + g.ny * k;
    s.c += s.xp * T(f.c1.at(loc));
    sh += double(s.xp) * f.c0.at(loc);
    s.xp = T(0);
  }
  if (j == 1) {
    const FaceDev& f = g.face[kBottom];
    const int loc = i + g.nx * k;
    s.c += s.ym * T(f.c1.at(loc));
    sh += double(s.ym) * f.c0.at(loc);
    s.ym = T(0);
  }
  if (j == g.ny - 2) {
    const FaceDev& f = g.face[kTop];
    const int loc = i + g.nx * k;
    s.c += s.yp * T(f.c1.at(loc));
    sh += double(s.yp) * f.c0.at(loc);
    s.yp = T(0);
  }
  if (d3) {
    if (k == 1) {
      const FaceDev& f = g.face[kFront];
      const int loc = i + g.nx * j;
      s.c += s.zm * T(f.c1.at(loc));
      sh += double(s.zm) * f.c0.at(loc);
      s.zm = T(0);
    }
    if (k == g.nz - 2) {
      const FaceDev& f = g.face[kBack];
      const int loc = i + g.nx * j;
      s.c += s.zp * T(f.c1.at(loc));
      sh += double(s.zp) * f.c0.at(loc);
      s.zp = T(0);
    }
  }
  if (bshift) *bshift = sh;
}

// Pointwise nonlinear terms sum(coeff * g(u)) (NonlinearTerm,
// include/pde_types.h:88-100), passed to kernels by value. nl_eval follows
// EvalNonlinear (src/backends/cpu/solvers/relaxation.cpp:27-45,
// src/backends/cpu/solver.cpp:234-256): terms summed in order, each product
// and sum rounded once (no contraction). Integer powers 0, 1 and 2 are exact
// or one rounding (u*u), which is what a correctly rounded pow gives.
constexpr int kMaxNonlinear = 8;
struct NonlinDev {
  int n;
  int kind[kMaxNonlinear];
  int power[kMaxNonlinear];
  double coeff[kMaxNonlinear];
};

__device__ __forceinline__ double nl_eval(const NonlinDev& nl, double u) {
  double v = 0.0;
  for (int t = 0; t < nl.n; ++t) {
    double gv;
    switch (nl.kind[t]) {
      case 0: {
        const int p = nl.power[t];
        gv = p == 0 ? 1.0 : p == 1 ? u : p == 2 ? __dmul_rn(u, u) : pow(u, double(p));
        break;
      }
      case 1: gv = sin(u); break;
      case 2: gv = cos(u); break;
      case 3: gv = exp(u); break;
      default: gv = fabs(u); break;
    }
    v = __dadd_rn(v, __dmul_rn(nl.coeff[t], gv));
  }
  return v;
}

// f + nonlinear(u) in the reference's order ((f + integral) + nonlinear, the
// integral term being absent here); plain f without terms.
__device__ __forceinline__ double f_plus_nl(double fv, const NonlinDev& nl, double u) {
  return nl.n ? __dadd_rn(fv, nl_eval(nl, u)) : fv;
}

// Neighbour sum in the reference's left-to-right order
// (src/backends/cpu/solver.cpp:892-898, cpu_utils.cpp:428-433).
template <typename T>
__device__ __forceinline__ T nb_sum(const Stencil<T>& s, T xp, T xm, T yp, T ym, T zp, T zm, int dim) {
  T v = s.xp * xp + s.xm * xm + s.yp * yp + s.ym * ym;
  if (dim == 3) v = v + s.zp * zp + s.zm * zm;
  return v;
}

// ---------------------------------------------------------------- reduction

constexpr int kMaxRed = 4;

// Block-wide sum of up to kMaxRed values; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red_smem[32][NV];
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
  const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
  const int warp = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
  const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) red_smem[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      v[q] = lane < nwarps ? red_smem[lane][q] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], off);
    }
  }
}

template <int NV>
__device__ __forceinline__ void block_max(double (&v)[NV]) {
  __shared__ double redm_smem[32][NV];
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[q] = fmax(v[q], __shfl_down_sync(0xffffffffu, v[q], off));
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, warp = tid >> 5;
  const int nwarps = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) redm_smem[warp][q] = v[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      v[q] = lane < nwarps ? redm_smem[lane][q] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v[q] = fmax(v[q], __shfl_down_sync(0xffffffffu, v[q], off));
    }
  }
}

// Grid reduction without a second launch: each block stores its partials, the
// last block to arrive (atomic ticket) sums them in block order, so the result
// is deterministic for a given launch shape. `post` runs in thread 0 of that
// last block with the totals (it derives Krylov scalars on the device).
struct RedSlot {
  double* partials;     // [nblocks * NV]
  unsigned* ticket;     // zero-initialised; reset by the last block
  double* out;          // [NV]
};

struct NoPost {
  __device__ void operator()(const double*) const {}
};

template <int NV, bool MAX, class Post>
__device__ __forceinline__ void grid_reduce(double (&v)[NV], const RedSlot& slot, const Post& post) {
  if (MAX)
    block_max<NV>(v);
  else
    block_sum<NV>(v);
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  __shared__ bool last_block;
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) slot.partials[(size_t)bid * NV + q] = v[q];
    __threadfence();
    const unsigned t = atomicAdd(slot.ticket, 1u);
    last_block = (t == nblocks - 1);
  }
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = MAX ? 0.0 : 0.0;
  for (unsigned b = tid; b < nblocks; b += nthreads)
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double pv = __ldcg(slot.partials + (size_t)b * NV + q);
      acc[q] = MAX ? fmax(acc[q], pv) : acc[q] + pv;
    }
  if (MAX)
    block_max<NV>(acc);
  else
    block_sum<NV>(acc);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) slot.out[q] = acc[q];
    post(acc);
    *slot.ticket = 0u;
  }
}

}  // namespace pdeb
