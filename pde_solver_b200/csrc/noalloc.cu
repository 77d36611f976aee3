// Jacobi solve that allocates nothing.
//
// Some callers cannot let a library allocate device memory: code that runs
// inside another runtime's fixed memory arena, hosts that forbid allocation
// after start-up (real-time loops), or plugins that must not touch the
// device allocator at all. pdeb200_jacobi_noalloc serves them: the caller
// passes device pointers for the inputs (f, k or nodal coefficients) and for
// the output field, and the solver's scratch (the second Jacobi field, the
// reduction partials and the control block) lives in one file-scope device
// array that every GPU loading the library holds until the process exits.
//
// Limits and sharing: the array holds kNoAllocMaxNodes nodes of the second
// field and kNoAllocMaxBlocks reduction slots, one per x-y block of 32 x 8
// columns, so a grid must have at most 1048576 nodes and
// ceil(nx/32)*ceil(ny/8) <= 8192 (a long, thin 2D grid can reach the second
// limit first); larger grids are rejected with PDEB200_ERR_UNSUPPORTED. Every
// call uses the same array. Calls that overlap on the GPU (two host threads,
// or two streams, at once) race on it and corrupt each other; the caller
// serialises them. Each call clears what must start at zero (the control
// block, the reduction tickets, the second field).
//
// Set-up: every call looks up the array's device address with
// cudaGetSymbolAddress while the device is current (the first call on a
// device also loads the module there, so it should come before any stream
// capture on that device). The address is not cached, so a device reset
// between calls is harmless.
#include <cstring>

#include "host.h"

namespace pdeb {

constexpr long long kNoAllocMaxNodes = 1LL << 20;  // second Jacobi field: 8 MiB
constexpr long long kNoAllocMaxBlocks = 8192;      // reduction partial slots
constexpr int kNoAllocDevices = 64;

struct NoAllocLayout {
  Ctl ctl;
  unsigned tickets[4];
  int degenerate;
  int pad;
  double redout[4 * kMaxRed];
  double partials[kNoAllocMaxBlocks * kMaxRed];
  double field[kNoAllocMaxNodes];
};

constexpr size_t kNoAllocBytes = (sizeof(NoAllocLayout) + 255) / 256 * 256;

// The scratch. In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

struct PostDeltaNA {
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

// Looked up on every call (with `device` current), not cached: after a
// cudaDeviceReset the module is loaded again and the array may move.
NoAllocLayout* scratch_for(int device) {
  (void)device;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw StatusFailure{PDEB200_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e)};
  }
  return static_cast<NoAllocLayout*>(p);
}

int launch_blocks(const dim3& g) { return (int)((long long)g.x * g.y * g.z); }

}  // namespace

static pdeb200_status jacobi_noalloc(const pdeb200_problem* p, int32_t max_iter_in, double tol, int32_t device,
                                     cudaStream_t stream, double* d_grid, pdeb200_report* rep) {
  if (!p || !d_grid) throw StatusFailure{PDEB200_ERR_INVALID, "null problem or output"};
  if (p->mem_space != PDEB200_MEM_DEVICE)
    throw StatusFailure{PDEB200_ERR_INVALID, "pdeb200_jacobi_noalloc takes device pointers (mem_space DEVICE)"};
  for (int f = 0; f < 6; ++f)
    if (p->face[f].value_arr || p->face[f].alpha_arr || p->face[f].beta_arr || p->face[f].gamma_arr)
      throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "pdeb200_jacobi_noalloc takes constant face values only"};
  const long long n = (long long)p->nx * p->ny * (p->nz > 1 ? p->nz : 1);
  if (n > kNoAllocMaxNodes)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "grid exceeds the 1048576-node limit of pdeb200_jacobi_noalloc"};
  if (device < 0 || device >= kNoAllocDevices) throw StatusFailure{PDEB200_ERR_INVALID, "device ordinal out of range"};
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device >= count) {
    cudaGetLastError();
    throw StatusFailure{PDEB200_ERR_NO_DEVICE, "CUDA device unavailable"};
  }
  int prev = 0;
  PDEB_CUDA(cudaGetDevice(&prev));
  PDEB_CUDA(cudaSetDevice(device));
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};

  NoAllocLayout* S = scratch_for(device);
  // problem descriptor: with device inputs and constant faces nothing is copied
  DevProblem P;
  upload_problem(nullptr, p, &P);
  const GridDev& g = P.g;
  const int max_iter = max_iter_in > 1 ? max_iter_in : 1;
  const dim3 grid = stencil_grid_auto(g), block = stencil_block();
  if (launch_blocks(grid) > kNoAllocMaxBlocks)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED,
                        "x-y plane too wide for pdeb200_jacobi_noalloc: ceil(nx/32)*ceil(ny/8) must be at most 8192"};
  if (P.coef_kind == kConst && std::fabs(P.cc.c) < 1e-12)
    throw StatusFailure{PDEB200_ERR_DEGENERATE, "degenerate PDE center coefficient"};

  // clear what must start at zero
  Ctl h{};
  h.max_iter = max_iter;
  h.tol = tol;
  h.status = PDEB200_ERR_NOT_CONVERGED;
  PDEB_CUDA(cudaMemcpyAsync(&S->ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
  PDEB_CUDA(cudaMemsetAsync(S->tickets, 0, sizeof(S->tickets) + sizeof(int) * 2, stream));
  PDEB_CUDA(cudaMemsetAsync(S->field, 0, sizeof(double) * n, stream));
  PDEB_CUDA(cudaMemsetAsync(d_grid, 0, sizeof(double) * n, stream));
  const RedSlot slot{S->partials, S->tickets, S->redout};
  double* buf[2] = {d_grid, S->field};
  const long long faces = 2LL * g.ny * g.nz + 2LL * g.nx * g.nz + (g.dim == 3 ? 2LL * g.nx * g.ny : 0);
  const int fb = (int)std::min<long long>((faces + 255) / 256, 1024);
  k_fill_boundary<<<fb, 256, 0, stream>>>(g, buf[0], &S->ctl, 1);
  int done_iters = 0;
  Ctl host{};
  int batch = 1;
  for (int t = 0; t < max_iter;) {
    for (int b = 0; b < batch && t < max_iter; ++b, ++t) {
      double* src = buf[t & 1];
      double* dst = buf[(t + 1) & 1];
      with_coef(P, [&](const auto& cf) {
        using Coef = std::decay_t<decltype(cf)>;
        k_jacobi<Coef, PostDeltaNA><<<grid, block, 0, stream>>>(g, cf, P.f, P.f_const, P.nl, src, dst, slot,
                                                                 PostDeltaNA{&S->ctl}, &S->ctl, &S->degenerate);
      });
      k_fill_boundary<<<fb, 256, 0, stream>>>(g, dst, &S->ctl, 1);
    }
    PDEB_CUDA(cudaMemcpyAsync(&host, &S->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
    PDEB_CUDA(cudaStreamSynchronize(stream));
    if (host.stop) break;
    batch = batch * 2 < 16 ? batch * 2 : 16;
  }
  PDEB_CUDA(cudaGetLastError());
  done_iters = host.iter;
  int degenerate = 0;
  PDEB_CUDA(cudaMemcpyAsync(&degenerate, &S->degenerate, sizeof(int), cudaMemcpyDeviceToHost, stream));
  if (done_iters & 1)
    PDEB_CUDA(cudaMemcpyAsync(d_grid, S->field, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
  PDEB_CUDA(cudaStreamSynchronize(stream));
  if (rep) {
    rep->iterations = done_iters;
    rep->last_delta = host.delta;
    rep->converged = host.status == PDEB200_OK;
  }
  if (degenerate) return PDEB200_ERR_DEGENERATE;
  return (pdeb200_status)host.status;
}

}  // namespace pdeb

extern "C" pdeb200_status pdeb200_jacobi_noalloc(const pdeb200_problem* prob, int32_t max_iter, double tol,
                                                 int32_t device, void* stream, double* out_grid,
                                                 pdeb200_report* report) {
  using namespace pdeb;
  if (report) std::memset(report, 0, sizeof(*report));
  try {
    return jacobi_noalloc(prob, max_iter, tol, device, static_cast<cudaStream_t>(stream), out_grid, report);
  } catch (const StatusFailure& s) {
    set_report_msg(report, s.what);
    return s.status;
  } catch (const CudaFailure& c) {
    set_report_msg(report, c.what);
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
}
