// Host-side runtime of libpdeb200: per-device contexts, stream-ordered device
// buffers, the device copy of a problem and the launch helpers shared by the
// solver drivers.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <mutex>
#include <utility>
#include <string>
#include <vector>

#include "../../include/pdeb200.h"
#include "kernels.cuh"

namespace pdeb {

struct Error {
  pdeb200_status status = PDEB200_OK;
  std::string msg;
};

#define PDEB_CUDA(call)                                                         \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) throw CudaFailure(e_, #call, __FILE__, __LINE__);    \
  } while (0)

struct CudaFailure {
  cudaError_t err;
  std::string what;
  CudaFailure(cudaError_t e, const char* call, const char* file, int line)
      : err(e), what(std::string(cudaGetErrorString(e)) + " at " + file + ":" + std::to_string(line) + " (" + call + ")") {}
};

struct StatusFailure {
  pdeb200_status status;
  std::string what;
};

// Device buffer from the device's stream-ordered memory pool. The pool keeps
// freed blocks (release threshold = max), so repeated solves of one shape do
// not go back to the driver.
class Buf {
 public:
  Buf() = default;
  Buf(size_t bytes, cudaStream_t s) : bytes_(bytes), s_(s) {
    if (bytes) {
      cudaError_t e = cudaMallocAsync(&p_, bytes, s);
      if (e == cudaErrorMemoryAllocation) throw StatusFailure{PDEB200_ERR_OOM, "device memory exhausted"};
      PDEB_CUDA(e);
    }
  }
  ~Buf() { reset(); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  Buf(Buf&& o) noexcept { *this = std::move(o); }
  Buf& operator=(Buf&& o) noexcept {
    if (this != &o) {
      reset();
      p_ = o.p_;
      bytes_ = o.bytes_;
      s_ = o.s_;
      o.p_ = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  void reset() {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    bytes_ = 0;
  }
  template <typename T>
  T* as() const { return static_cast<T*>(p_); }
  size_t bytes() const { return bytes_; }

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
  cudaStream_t s_ = nullptr;
};

struct ProfPending {
  std::string name;
  cudaEvent_t a, b;
  double bytes;
};

struct ProfStat {
  std::string name;
  long long launches = 0;
  double total_ms = 0.0;
  double bytes = 0.0;
};

struct Context {
  int dev = 0;
  cudaStream_t stream = nullptr;      // launch stream in use
  cudaStream_t own_stream = nullptr;  // the library's own stream
  bool prof = false;
  std::vector<ProfPending> pending;
  std::vector<ProfStat> stats;
  std::vector<cudaEvent_t> evpool;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Ctl* d_ctl = nullptr;     // device control block
  Ctl* h_ctl = nullptr;     // pinned mirror
  double* d_partials = nullptr;
  unsigned* d_tickets = nullptr;
  double* d_redout = nullptr;
  size_t max_blocks = 0;
  int num_sms = 148;
  bool pdl = true;  // launch_dep launches carry programmatic stream serialization
  std::string name;
  std::mutex mu;
  long long launches = 0;
  std::shared_ptr<void> io_staging;  // output staging buffers, kept between writes (vtk.cu)

  cudaEvent_t ev_get() {
    if (!evpool.empty()) {
      cudaEvent_t e = evpool.back();
      evpool.pop_back();
      return e;
    }
    cudaEvent_t e;
    PDEB_CUDA(cudaEventCreate(&e));
    return e;
  }
  // accumulate pending kernel timings (after the stream has been synchronised)
  void prof_flush() {
    for (auto& p : pending) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
        ProfStat* st = nullptr;
        for (auto& s : stats)
          if (s.name == p.name && s.bytes == p.bytes) st = &s;
        if (!st) {
          stats.push_back(ProfStat{p.name, 0, 0.0, p.bytes});
          st = &stats.back();
        }
        st->launches += 1;
        st->total_ms += ms;
      }
      evpool.push_back(p.a);
      evpool.push_back(p.b);
    }
    pending.clear();
  }

  RedSlot slot(int which = 0) const {
    return RedSlot{d_partials + (size_t)which * max_blocks * kMaxRed, d_tickets + which, d_redout + which * kMaxRed};
  }
  void count(int n = 1) { launches += n; }
};

// Brackets one launch with events on the launch stream while profiling is on.
// Names carry the MG level ("rbgs_color_pass@L0"); level -1 = no level.
struct ProfScope {
  Context* c;
  std::string name;
  double bytes;
  cudaEvent_t a = nullptr;
  ProfScope(Context* ctx, const char* n, int level, double b) : c(ctx), bytes(b) {
    if (c->prof) {
      name = level >= 0 ? std::string(n) + "@L" + std::to_string(level) : std::string(n);
      a = c->ev_get();
      PDEB_CUDA(cudaEventRecord(a, c->stream));
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEvent_t b = c->ev_get();
      cudaEventRecord(b, c->stream);
      c->pending.push_back(ProfPending{name, a, b, bytes});
    }
  }
};

inline double interior_dofs(const GridDev& g) {
  return double(g.nx - 2) * double(g.ny - 2) * double(g.dim == 3 ? g.nz - 2 : 1);
}

Context* get_context(int dev);  // throws StatusFailure / CudaFailure
// A context of one's own (stream, control block, reduction buffers): callers
// that run solves concurrently on one device give each thread its own.
void init_context(Context* c, int dev);
void free_context(Context* c);
void release_contexts();

// Device copy of a problem, with face closures materialised.
struct DevProblem {
  GridDev g{};
  int coef_kind = 0;
  CoefConst cc{};
  CoefDivk<double> cd{};
  CoefNodal cn{};
  const double* f = nullptr;
  double f_const = 0.0;
  const double* u0 = nullptr;
  NonlinDev nl{};  // pointwise nonlinear terms (relaxation, time series, 2D residual norms)
  double dx = 0, dy = 0, dz = 0;
  double a = 0, b = 0, az = 0, c = 0, d = 0, dzc = 0, e = 0, ut = 0;
  std::vector<Buf> owned;
  bool device_inputs = false;
};

// Validates and uploads; host arrays of the problem are copied on ctx->stream.
void upload_problem(Context* ctx, const pdeb200_problem* p, DevProblem* out);
// Validation, geometry, faces and coefficient scalars only: f, u0, k and
// nodal stay unset (the caller places them).
void describe_problem(Context* ctx, const pdeb200_problem* p, DevProblem* out);

// Builds the face parameters of `g` for spacing (dx,dy,dz) from the host face
// descriptions; arrays are sampled with `stride` (1 on the finest level, 2^l
// on level l) and uploaded into `owned`.
void build_faces(Context* ctx, const pdeb200_problem* p, int nx, int ny, int nz, double dx, double dy, double dz,
                 int stride, GridDev* g, std::vector<Buf>* owned);

CoefConst make_const(double a, double b, double az, double c, double d, double dz, double e, double dx, double dy,
                     double dzs, int dim);

inline dim3 stencil_block() { return dim3(kBx, kBy, 1); }
dim3 stencil_grid(const GridDev& g, int zchunk = 16);
dim3 stencil_grid_full(const GridDev& g, int zchunk = 16);
// z-chunking chosen for occupancy: about kTargetBlocks blocks, at least one
// interior plane per thread
dim3 stencil_grid_auto(const GridDev& g, long long target_blocks = 0);
// launch shape of the colour passes (k_rbgs): on levels larger than L2 about
// three waves of the three blocks per SM their registers allow (faster than
// the default target)
inline dim3 rbgs_grid(const GridDev& g) {
  // levels that fit in L2 (129^3 and below) launch one wave of 148 x 3 blocks:
  // 129^3 14.6 -> 13.8 us and 65^3 4.3 -> 3.9 us per pass in a replayed graph,
  // 257^3 solve 21.93 -> 21.8 ms, 129^3 6.2 -> 6.0 ms, 65^3 3.2 -> 3.1 ms
  return stencil_grid_auto(g, g.n > (1LL << 22) ? 148 * 9 : 148 * 3);
}
// launch shape of the fused red-black sweep (64 x 8 column tiles)
dim3 fused_grid(const GridDev& g);
// launch shape of the marching single-pass sweep (64 x 8 interior column tiles, z chunks)
dim3 march_grid(const GridDev& g);
// launch shape of the staged single-pass sweep (32 x 8 column tiles, z chunks
// for about four resident blocks per SM over two waves)
dim3 sweep_grid(const GridDev& g);
inline int vec_blocks(long long n, const Context* ctx) {
  long long b = (n + 255) / 256;
  long long cap = (long long)ctx->num_sms * 8;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// Launch of a kernel that calls ctl_skip_dep() before its first memory access,
// with programmatic stream serialization when ctx->pdl is set: the launch may
// be scheduled while the previous kernel of the stream drains, and waits in
// ctl_skip_dep until that kernel has completed. Inside a captured graph this
// becomes a programmatic edge. The arguments are those of the kernel in full
// (no defaulted parameters).
template <typename... KArgs, typename... Args>
inline void launch_dep(const Context* ctx, dim3 grid, dim3 block, size_t smem, void (*kern)(KArgs...),
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = ctx->pdl ? 1 : 0;
  PDEB_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// Dispatch on the coefficient form of a DevProblem: fn(coef) with the concrete type.
template <class Fn>
void with_coef(const DevProblem& P, Fn&& fn) {
  switch (P.coef_kind) {
    case kDivk: fn(P.cd); break;
    case kNodal: fn(P.cn); break;
    default: fn(P.cc); break;
  }
}

void set_report_msg(pdeb200_report* r, const std::string& m);

// Solver drivers (solvers.cu)
pdeb200_status solve_dispatch(Context* ctx, DevProblem& P, const pdeb200_problem* hp, const pdeb200_options* o,
                              double* d_out, pdeb200_report* rep);
// Host-array entry bodies on a given context (the caller serialises use of ctx).
pdeb200_status solve_on(Context* ctx, const pdeb200_problem* prob, const pdeb200_options* opt, double* out_grid,
                        pdeb200_report* report);
pdeb200_status time_series_on(Context* ctx, const pdeb200_problem* prob, const pdeb200_time_options* topt,
                              pdeb200_frame_cb on_frame, void* user, double* out_grid, pdeb200_report* report);
pdeb200_status residual_norms_dev(Context* ctx, DevProblem& P, const double* d_grid, double* l2, double* linf);
pdeb200_status apply_dev(Context* ctx, DevProblem& P, const double* d_x, double* d_y);
pdeb200_status time_series_dev(Context* ctx, DevProblem& P, const pdeb200_time_options* t, pdeb200_frame_cb cb,
                               void* user, bool host_frames, double* d_out, pdeb200_report* rep);
pdeb200_status project_dev(Context* ctx, int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                           double* u, double* v, double* w, double* p, const pdeb200_projection_options* po,
                           pdeb200_projection_report* rep);

}  // namespace pdeb
