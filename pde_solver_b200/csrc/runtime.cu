// Runtime of libpdeb200: device contexts, problem upload, face closures and
// the extern "C" entry points declared in include/pdeb200.h.
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <limits>

#include "host.h"
#include "march.cuh"

namespace pdeb {

namespace {
std::mutex g_ctx_mu;
std::vector<std::unique_ptr<Context>> g_ctx;
}  // namespace

Context* get_context(int dev) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    throw StatusFailure{PDEB200_ERR_NO_DEVICE, e != cudaSuccess ? std::string("cudaGetDeviceCount failed: ") +
                                                                      cudaGetErrorString(e)
                                                                : "no CUDA devices found"};
  }
  if (dev < 0 || dev >= count) throw StatusFailure{PDEB200_ERR_INVALID, "device ordinal out of range"};
  if ((int)g_ctx.size() < count) g_ctx.resize(count);
  PDEB_CUDA(cudaSetDevice(dev));
  if (!g_ctx[dev]) {
    auto c = std::make_unique<Context>();
    init_context(c.get(), dev);
    g_ctx[dev] = std::move(c);
  }
  return g_ctx[dev].get();
}

void init_context(Context* c, int dev) {
  PDEB_CUDA(cudaSetDevice(dev));
  c->dev = dev;
  cudaDeviceProp prop;
  PDEB_CUDA(cudaGetDeviceProperties(&prop, dev));
  c->name = prop.name;
  c->num_sms = prop.multiProcessorCount;
  c->pdl = std::getenv("PDEB200_NO_PDL") == nullptr;
  PDEB_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = c->own_stream;
  PDEB_CUDA(cudaEventCreate(&c->ev0));
  PDEB_CUDA(cudaEventCreate(&c->ev1));
  PDEB_CUDA(cudaMalloc(&c->d_ctl, sizeof(Ctl)));
  PDEB_CUDA(cudaMallocHost(&c->h_ctl, sizeof(Ctl)));
  c->max_blocks = kMaxGridBlocks;
  const int nslots = 4;
  PDEB_CUDA(cudaMalloc(&c->d_partials, sizeof(double) * c->max_blocks * kMaxRed * nslots));
  PDEB_CUDA(cudaMalloc(&c->d_tickets, sizeof(unsigned) * nslots));
  PDEB_CUDA(cudaMemset(c->d_tickets, 0, sizeof(unsigned) * nslots));
  PDEB_CUDA(cudaMalloc(&c->d_redout, sizeof(double) * kMaxRed * nslots));
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = std::numeric_limits<uint64_t>::max();
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
}

void free_context(Context* c) {
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->stream);
  c->io_staging.reset();
  cudaFree(c->d_ctl);
  cudaFreeHost(c->h_ctl);
  cudaFree(c->d_partials);
  cudaFree(c->d_tickets);
  cudaFree(c->d_redout);
  cudaEventDestroy(c->ev0);
  cudaEventDestroy(c->ev1);
  for (auto e : c->evpool) cudaEventDestroy(e);
  c->evpool.clear();
  cudaStreamDestroy(c->own_stream);
  c->d_ctl = nullptr;
  c->h_ctl = nullptr;
  c->d_partials = nullptr;
  c->d_tickets = nullptr;
  c->d_redout = nullptr;
  c->own_stream = c->stream = nullptr;
}

void release_contexts() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  for (auto& c : g_ctx) {
    if (!c) continue;
    free_context(c.get());
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, c->dev) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    c.reset();
  }
}

// Stencil launch shapes. The number of blocks never exceeds kMaxGridBlocks,
// the capacity of the reduction partial buffers (upload_problem rejects grids
// whose x-y tiling alone would exceed it).
static int cap_chunks(long long xy_blocks, int chunks) {
  const long long cap = kMaxGridBlocks / (xy_blocks > 0 ? xy_blocks : 1);
  if (chunks > cap) chunks = (int)(cap > 0 ? cap : 1);
  return chunks > 0 ? chunks : 1;
}

dim3 stencil_grid(const GridDev& g, int zchunk) {
  const int kint = g.dim == 3 ? g.nz - 2 : 1;
  const int chunks = g.dim == 3 ? (kint + zchunk - 1) / zchunk : 1;
  const dim3 xy((g.nx + kBx - 1) / kBx, (g.ny + kBy - 1) / kBy, 1);
  return dim3(xy.x, xy.y, cap_chunks((long long)xy.x * xy.y, chunks));
}

dim3 stencil_grid_auto(const GridDev& g, long long target_blocks) {
  const long long kTargetBlocks = target_blocks > 0 ? target_blocks : 148 * 16;
  const int kint = g.dim == 3 ? g.nz - 2 : 1;
  const dim3 xy((g.nx + kBx - 1) / kBx, (g.ny + kBy - 1) / kBy, 1);
  const long long xyb = (long long)xy.x * xy.y;
  long long chunks = (kTargetBlocks + xyb - 1) / xyb;
  if (chunks > kint) chunks = kint;
  if (chunks < 1) chunks = 1;
  return dim3(xy.x, xy.y, cap_chunks(xyb, (int)chunks));
}

dim3 sweep_grid(const GridDev& g) {
  const long long kTargetBlocks = 148 * 8;
  const int kint = g.dim == 3 ? g.nz - 2 : 1;
  const dim3 xy((g.nx + 31) / 32, (g.ny + 7) / 8, 1);
  const long long xyb = (long long)xy.x * xy.y;
  long long chunks = (kTargetBlocks + xyb - 1) / xyb;
  // at least 16 planes per chunk so the two staging planes are amortised
  const long long max_chunks = (kint + 15) / 16;
  if (chunks > max_chunks) chunks = max_chunks;
  if (chunks < 1) chunks = 1;
  return dim3(xy.x, xy.y, cap_chunks(xyb, (int)chunks));
}

dim3 fused_grid(const GridDev& g) {
  const long long kTargetBlocks = 148 * 8;
  const int kint = g.dim == 3 ? g.nz - 2 : 1;
  const dim3 xy((g.nx + kFx - 1) / kFx, (g.ny + kBy - 1) / kBy, 1);
  const long long xyb = (long long)xy.x * xy.y;
  long long chunks = (kTargetBlocks + xyb - 1) / xyb;
  // at least two slabs per chunk so the halo planes are amortised
  const long long max_chunks = (kint + 2 * kSlab - 1) / (2 * kSlab);
  if (chunks > max_chunks) chunks = max_chunks;
  if (chunks < 1) chunks = 1;
  return dim3(xy.x, xy.y, cap_chunks(xyb, (int)chunks));
}

dim3 march_grid(const GridDev& g) {
  // about `waves` waves of the two resident blocks per SM its shared memory
  // allows, at least 16 planes per chunk (each chunk re-reads 3 planes)
  static const int waves = [] {
    const char* e = std::getenv("PDEB200_MARCH_WAVES");
    const int w = e ? std::atoi(e) : 3;
    return w > 0 ? w : 3;
  }();
  const long long target = 148LL * 2 * waves;
  const int kint = g.nz - 2;
  const dim3 xy((g.nx - 2 + kMTx - 1) / kMTx, (g.ny - 2 + kMTy - 1) / kMTy, 1);
  const long long xyb = (long long)xy.x * xy.y;
  long long chunks = (target + xyb - 1) / xyb;
  const long long max_chunks = (kint + 15) / 16;
  if (chunks > max_chunks) chunks = max_chunks;
  if (chunks < 1) chunks = 1;
  return dim3(xy.x, xy.y, (unsigned)chunks);
}

dim3 stencil_grid_full(const GridDev& g, int zchunk) {
  const int chunks = (g.nz + zchunk - 1) / zchunk;
  const dim3 xy((g.nx + kBx - 1) / kBx, (g.ny + kBy - 1) / kBy, 1);
  return dim3(xy.x, xy.y, cap_chunks((long long)xy.x * xy.y, chunks));
}

// The reference's constant stencil (src/backends/cpu/solver.cpp:723-729,
// cpu_utils.cpp:290-294), evaluated on the host in the same order.
CoefConst make_const(double a, double b, double az, double c, double d, double dz, double e, double dx, double dy,
                     double dzs, int dim) {
  CoefConst k{};
  const double ax = a / (dx * dx);
  const double by = b / (dy * dy);
  const double cx = c / (2.0 * dx);
  const double dyc = d / (2.0 * dy);
  k.xp = ax + cx;
  k.xm = ax - cx;
  k.yp = by + dyc;
  k.ym = by - dyc;
  if (dim == 3) {
    const double cz = az / (dzs * dzs);
    const double dzc = dz / (2.0 * dzs);
    k.zp = cz + dzc;
    k.zm = cz - dzc;
    k.c = -2.0 * ax - 2.0 * by - 2.0 * cz + e;
  } else {
    k.zp = k.zm = 0.0;
    k.c = -2.0 * ax - 2.0 * by + e;
  }
  return k;
}

namespace {

Buf upload(Context* ctx, const void* host, size_t bytes) {
  Buf b(bytes, ctx->stream);
  PDEB_CUDA(cudaMemcpyAsync(b.as<void>(), host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return b;
}

// face dims in face-local order (first index fastest)
void face_dims(int f, int nx, int ny, int nz, int* w, int* hgt) {
  if (f <= kRight) {
    *w = ny;
    *hgt = nz;
  } else if (f <= kTop) {
    *w = nx;
    *hgt = nz;
  } else {
    *w = nx;
    *hgt = ny;
  }
}

}  // namespace

void build_faces(Context* ctx, const pdeb200_problem* p, int nx, int ny, int nz, double dx, double dy, double dz,
                 int stride, GridDev* g, std::vector<Buf>* owned) {
  const int dim = p->nz > 1 ? 3 : 2;
  const int fnx = p->nx, fny = p->ny, fnz = p->nz > 1 ? p->nz : 1;
  for (int f = 0; f < 6; ++f) {
    const pdeb200_face& hf = p->face[f];
    FaceDev& F = g->face[f];
    F.kind = hf.kind;
    F.active = (dim == 3 || f < kFront) ? 1 : 0;
    F.h = f <= kRight ? dx : (f <= kTop ? dy : dz);
    int w, hgt, fw, fh;
    face_dims(f, nx, ny, nz, &w, &hgt);
    face_dims(f, fnx, fny, fnz, &fw, &fh);
    const int cnt = w * hgt;
    // coarse face node -> nearest fine face node (stride 2^l for odd sizes)
    auto nearest = [](int a, int wc, int wf) -> long long {
      if (wc <= 1) return 0;
      return ((long long)a * (wf - 1) + (wc - 1) / 2) / (wc - 1);
    };
    auto sample = [&](const double* arr, std::vector<double>* out) {
      out->resize(cnt);
      for (int b = 0; b < hgt; ++b)
        for (int a = 0; a < w; ++a) {
          long long fi = stride == 1 ? a : nearest(a, w, fw);
          long long fj = stride == 1 ? b : nearest(b, hgt, fh);
          if (fi >= fw) fi = fw - 1;
          if (fj >= fh) fj = fh - 1;
          (*out)[(size_t)b * w + a] = arr[fj * fw + fi];
        }
    };
    const double* arrs[4] = {hf.value_arr, hf.alpha_arr, hf.beta_arr, hf.gamma_arr};
    const double scal[4] = {hf.value, hf.alpha, hf.beta, hf.gamma};
    FaceParam* params[4] = {&F.val, &F.alpha, &F.beta, &F.gamma};
    std::vector<double> host[4];
    bool any_arr = false;
    for (int q = 0; q < 4; ++q) {
      params[q]->s = scal[q];
      params[q]->a = nullptr;
      if (arrs[q] && F.active) {
        sample(arrs[q], &host[q]);
        owned->push_back(upload(ctx, host[q].data(), sizeof(double) * cnt));
        params[q]->a = owned->back().as<double>();
        any_arr = true;
      }
    }
    // folded closure u_b = c0 + c1 u_nb
    auto c01 = [&](double val, double al, double be, double ga, double* c0, double* c1) {
      const int is_max = f & 1;
      if (F.kind == kDirichlet) {
        *c0 = val;
        *c1 = 0.0;
      } else if (F.kind == kNeumann) {
        *c0 = is_max ? F.h * val : -F.h * val;
        *c1 = 1.0;
      } else {
        const double bh = be / F.h;
        const double den = is_max ? al - bh : al + bh;
        if (std::fabs(den) > 1e-12) {
          *c0 = ga / den;
          *c1 = (is_max ? -bh : bh) / den;
        } else {
          *c0 = 0.0;
          *c1 = 0.0;
        }
      }
    };
    if (!any_arr) {
      c01(hf.value, hf.alpha, hf.beta, hf.gamma, &F.c0.s, &F.c1.s);
      F.c0.a = F.c1.a = nullptr;
    } else {
      std::vector<double> c0(cnt), c1(cnt);
      for (int q = 0; q < cnt; ++q) {
        const double v[4] = {arrs[0] ? host[0][q] : scal[0], arrs[1] ? host[1][q] : scal[1],
                             arrs[2] ? host[2][q] : scal[2], arrs[3] ? host[3][q] : scal[3]};
        c01(v[0], v[1], v[2], v[3], &c0[q], &c1[q]);
      }
      owned->push_back(upload(ctx, c0.data(), sizeof(double) * cnt));
      F.c0.a = owned->back().as<double>();
      owned->push_back(upload(ctx, c1.data(), sizeof(double) * cnt));
      F.c1.a = owned->back().as<double>();
      F.c0.s = F.c1.s = 0.0;
    }
  }
}

void upload_problem(Context* ctx, const pdeb200_problem* p, DevProblem* P) {
  describe_problem(ctx, p, P);
  const long long n = P->g.n;
  auto take = [&](const double* ptr, size_t count) -> const double* {
    if (!ptr) return nullptr;
    if (P->device_inputs) return ptr;
    P->owned.push_back(upload(ctx, ptr, sizeof(double) * count));
    return P->owned.back().as<double>();
  };
  P->f = take(p->f, n);
  P->u0 = take(p->u0, n);
  if (p->coef_kind == PDEB200_COEF_DIVK) P->cd.k = take(p->k, n);
  if (p->coef_kind == PDEB200_COEF_NODAL) P->cn.nodal = take(p->nodal, 7 * n);
}

void describe_problem(Context* ctx, const pdeb200_problem* p, DevProblem* P) {
  if (!p) throw StatusFailure{PDEB200_ERR_INVALID, "null problem"};
  const int dim = p->nz > 1 ? 3 : 2;
  if (p->nx < 3 || p->ny < 3 || (dim == 3 && p->nz < 3))
    throw StatusFailure{PDEB200_ERR_INVALID, "grid must be at least 3 nodes per dimension"};
  if (!(p->xmax > p->xmin) || !(p->ymax > p->ymin) || (dim == 3 && !(p->zmax > p->zmin)))
    throw StatusFailure{PDEB200_ERR_INVALID, "domain bounds are invalid"};
  const long long n = (long long)p->nx * p->ny * (dim == 3 ? p->nz : 1);
  if (n > (1LL << 34)) throw StatusFailure{PDEB200_ERR_INVALID, "grid too large"};
  if ((long long)((p->nx + kBx - 1) / kBx) * ((p->ny + kBy - 1) / kBy) > kMaxGridBlocks)
    throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "x-y plane too large for one launch tiling"};
  for (int f = 0; f < 6; ++f)
    if (p->face[f].kind < 0 || p->face[f].kind > 2) throw StatusFailure{PDEB200_ERR_INVALID, "unknown boundary kind"};
  GridDev& g = P->g;
  g.nx = p->nx;
  g.ny = p->ny;
  g.nz = dim == 3 ? p->nz : 1;
  g.dim = dim;
  g.n = n;
  g.sxy = (long long)g.nx * g.ny;
  P->dx = (p->xmax - p->xmin) / (double)(g.nx - 1);
  P->dy = (p->ymax - p->ymin) / (double)(g.ny - 1);
  P->dz = dim == 3 ? (p->zmax - p->zmin) / (double)(g.nz - 1) : 0.0;
  P->a = p->a;
  P->b = p->b;
  P->az = p->az;
  P->c = p->c;
  P->d = p->d;
  P->dzc = p->dz;
  P->e = p->e;
  P->ut = p->ut;
  P->coef_kind = p->coef_kind;
  P->f_const = p->f_const;
  P->device_inputs = p->mem_space == PDEB200_MEM_DEVICE;
  if (p->n_nonlinear < 0 || p->n_nonlinear > PDEB200_MAX_NONLINEAR || (p->n_nonlinear > 0 && !p->nonlinear))
    throw StatusFailure{PDEB200_ERR_INVALID, "nonlinear terms: at most 8, with a term array"};
  P->nl = NonlinDev{};
  P->nl.n = p->n_nonlinear;
  for (int t = 0; t < p->n_nonlinear; ++t) {
    const pdeb200_nonlinear_term& nt = p->nonlinear[t];
    if (nt.kind < PDEB200_NL_POWER || nt.kind > PDEB200_NL_ABS)
      throw StatusFailure{PDEB200_ERR_INVALID, "unknown nonlinear term kind"};
    P->nl.kind[t] = nt.kind;
    P->nl.power[t] = nt.power;
    P->nl.coeff[t] = nt.coeff;
  }
  build_faces(ctx, p, g.nx, g.ny, g.nz, P->dx, P->dy, P->dz, 1, &g, &P->owned);
  switch (p->coef_kind) {
    case PDEB200_COEF_CONST:
      P->cc = make_const(p->a, p->b, p->az, p->c, p->d, p->dz, p->e, P->dx, P->dy, P->dz, dim);
      break;
    case PDEB200_COEF_DIVK: {
      if (!p->k) throw StatusFailure{PDEB200_ERR_INVALID, "COEF_DIVK needs k"};
      P->cd.k = nullptr;
      P->cd.ihx2 = 1.0 / (P->dx * P->dx);
      P->cd.ihy2 = 1.0 / (P->dy * P->dy);
      P->cd.ihz2 = dim == 3 ? 1.0 / (P->dz * P->dz) : 0.0;
      P->cd.cx = p->c / (2.0 * P->dx);
      P->cd.dyc = p->d / (2.0 * P->dy);
      P->cd.dzc = dim == 3 ? p->dz / (2.0 * P->dz) : 0.0;
      P->cd.e = p->e;
      break;
    }
    case PDEB200_COEF_NODAL: {
      if (!p->nodal) throw StatusFailure{PDEB200_ERR_INVALID, "COEF_NODAL needs nodal arrays"};
      P->cn.nodal = nullptr;
      P->cn.n = n;
      P->cn.dx2 = P->dx * P->dx;
      P->cn.dy2 = P->dy * P->dy;
      P->cn.dz2 = P->dz * P->dz;
      P->cn.tdx = 2.0 * P->dx;
      P->cn.tdy = 2.0 * P->dy;
      P->cn.tdz = 2.0 * P->dz;
      break;
    }
    default:
      throw StatusFailure{PDEB200_ERR_INVALID, "unknown coefficient kind"};
  }
}

pdeb200_status solve_on(Context* ctx, const pdeb200_problem* prob, const pdeb200_options* opt, double* out_grid,
                        pdeb200_report* report) {
  ctx->launches = 0;
  DevProblem P;
  upload_problem(ctx, prob, &P);
  const long long n = P.g.n;
  double* d_out = out_grid;
  Buf out_buf;
  if (!P.device_inputs) {
    out_buf = Buf(sizeof(double) * n, ctx->stream);
    d_out = out_buf.as<double>();
  }
  pdeb200_status s = solve_dispatch(ctx, P, prob, opt, d_out, report);
  if (!P.device_inputs && (s == PDEB200_OK || s == PDEB200_ERR_NOT_CONVERGED))
    PDEB_CUDA(cudaMemcpyAsync(out_grid, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
  PDEB_CUDA(cudaGetLastError());
  ctx->prof_flush();
  if (report) report->kernel_launches = (int32_t)ctx->launches;
  return s;
}

pdeb200_status time_series_on(Context* ctx, const pdeb200_problem* prob, const pdeb200_time_options* topt,
                              pdeb200_frame_cb on_frame, void* user, double* out_grid, pdeb200_report* report) {
  ctx->launches = 0;
  DevProblem P;
  upload_problem(ctx, prob, &P);
  const long long n = P.g.n;
  double* d_out = out_grid;
  Buf ob;
  if (!P.device_inputs) {
    ob = Buf(sizeof(double) * n, ctx->stream);
    d_out = ob.as<double>();
  }
  pdeb200_status s = time_series_dev(ctx, P, topt, on_frame, user, !P.device_inputs, d_out, report);
  if (!P.device_inputs && s == PDEB200_OK)
    PDEB_CUDA(cudaMemcpyAsync(out_grid, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
  if (report) report->kernel_launches = (int32_t)ctx->launches;
  return s;
}

void set_report_msg(pdeb200_report* r, const std::string& m) {
  if (!r) return;
  std::strncpy(r->message, m.c_str(), sizeof(r->message) - 1);
  r->message[sizeof(r->message) - 1] = '\0';
}

}  // namespace pdeb

using namespace pdeb;

namespace {

template <class Fn>
pdeb200_status guarded(pdeb200_report* rep, Fn&& fn) {
  try {
    return fn();
  } catch (const StatusFailure& s) {
    set_report_msg(rep, s.what);
    return s.status;
  } catch (const CudaFailure& c) {
    set_report_msg(rep, c.what);
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    set_report_msg(rep, "host memory exhausted");
    return PDEB200_ERR_OOM;
  }
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

int32_t pdeb200_abi_version(void) { return PDEB200_ABI_VERSION; }

int32_t pdeb200_probe(char* note, size_t note_len) {
  int count = 0;
  cudaError_t err = cudaGetDeviceCount(&count);
  std::string msg;
  int ok = 0;
  if (err != cudaSuccess || count == 0) {
    msg = err != cudaSuccess ? std::string("cudaGetDeviceCount failed: ") + cudaGetErrorString(err)
                             : "no CUDA devices found";
    cudaGetLastError();
  } else {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) == cudaSuccess) msg = std::string("device: ") + prop.name;
    ok = 1;
  }
  if (note && note_len) {
    std::strncpy(note, msg.c_str(), note_len - 1);
    note[note_len - 1] = '\0';
  }
  return ok;
}

const char* pdeb200_status_string(int32_t s) {
  switch (s) {
    case PDEB200_OK: return "";
    case PDEB200_ERR_INVALID: return "invalid input";
    case PDEB200_ERR_UNSUPPORTED: return "selected solve not supported by the B200 backend";
    case PDEB200_ERR_NO_DEVICE: return "CUDA unavailable";
    case PDEB200_ERR_CUDA: return "CUDA error";
    case PDEB200_ERR_OOM: return "device memory exhausted";
    case PDEB200_ERR_NOT_CONVERGED: return "solver failed to converge";
    case PDEB200_ERR_BREAKDOWN: return "Krylov breakdown";
    case PDEB200_ERR_DEGENERATE: return "degenerate PDE center coefficient";
    case PDEB200_ERR_CANCELLED: return "solve cancelled";
    case PDEB200_ERR_TIMEOUT: return "device wait timed out";
    case PDEB200_ERR_BUSY: return "server busy";
    default: return "unknown status";
  }
}

void pdeb200_default_options(pdeb200_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->method = PDEB200_JACOBI;
  o->max_iter = 10000;
  o->tol = 1e-6;
  o->tol_mode = PDEB200_TOL_REFERENCE;
  o->precision = PDEB200_FP64;
  o->sor_omega = 1.5;
  o->gmres_restart = 30;
  o->mg_pre_smooth = 2;
  o->mg_post_smooth = 2;
  o->mg_coarse_iters = 50;
  o->mg_max_levels = 10;
  o->gs_ordering = PDEB200_ORDER_LEXICOGRAPHIC;
  o->device = 0;
  o->check_interval = 0;
  o->inner_tol = 1e-5;
  o->bf16_coefficients = 0;
  o->max_outer = 50;
  o->cancel = nullptr;
}

void pdeb200_release_all(void) { release_contexts(); }

pdeb200_status pdeb200_set_stream(int32_t device, void* stream) {
  return guarded(nullptr, [&]() -> pdeb200_status {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return PDEB200_OK;
  });
}

void pdeb200_profile_enable(int32_t device, int32_t on) {
  guarded(nullptr, [&]() -> pdeb200_status {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->prof = on != 0;
    if (on) ctx->stats.clear();
    return PDEB200_OK;
  });
}

int32_t pdeb200_profile_read(int32_t device, pdeb200_kernel_stat* stats, int32_t max_stats) {
  int32_t count = 0;
  guarded(nullptr, [&]() -> pdeb200_status {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    count = (int32_t)ctx->stats.size();
    for (int32_t q = 0; q < count && q < max_stats && stats; ++q) {
      std::memset(&stats[q], 0, sizeof(stats[q]));
      std::strncpy(stats[q].name, ctx->stats[q].name.c_str(), sizeof(stats[q].name) - 1);
      stats[q].launches = ctx->stats[q].launches;
      stats[q].total_ms = ctx->stats[q].total_ms;
      stats[q].bytes_per_launch = ctx->stats[q].bytes;
    }
    return PDEB200_OK;
  });
  return count;
}

pdeb200_status pdeb200_solve(const pdeb200_problem* prob, const pdeb200_options* opt, double* out_grid,
                             pdeb200_report* report) {
  const double t0 = now_ms();
  if (report) std::memset(report, 0, sizeof(*report));
  if (!prob || !opt || !out_grid) {
    set_report_msg(report, "null argument");
    return PDEB200_ERR_INVALID;
  }
  pdeb200_status st = guarded(report, [&]() -> pdeb200_status {
    Context* ctx = get_context(opt->device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    return solve_on(ctx, prob, opt, out_grid, report);
  });
  if (report) {
    report->total_ms = now_ms() - t0;
    if (st != PDEB200_OK && report->message[0] == '\0') set_report_msg(report, pdeb200_status_string(st));
  }
  return st;
}

pdeb200_status pdeb200_residual_norms(const pdeb200_problem* prob, const double* grid, int32_t device, double* l2,
                                      double* linf) {
  if (!prob || !grid || !l2 || !linf) return PDEB200_ERR_INVALID;
  return guarded(nullptr, [&]() -> pdeb200_status {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    DevProblem P;
    upload_problem(ctx, prob, &P);
    const double* d_grid = grid;
    Buf gb;
    if (!P.device_inputs) {
      gb = Buf(sizeof(double) * P.g.n, ctx->stream);
      PDEB_CUDA(cudaMemcpyAsync(gb.as<double>(), grid, sizeof(double) * P.g.n, cudaMemcpyHostToDevice, ctx->stream));
      d_grid = gb.as<double>();
    }
    pdeb200_status s = residual_norms_dev(ctx, P, d_grid, l2, linf);
    PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
    return s;
  });
}

pdeb200_status pdeb200_apply(const pdeb200_problem* prob, const double* x, double* y, int32_t device) {
  if (!prob || !x || !y) return PDEB200_ERR_INVALID;
  return guarded(nullptr, [&]() -> pdeb200_status {
    Context* ctx = get_context(device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    DevProblem P;
    upload_problem(ctx, prob, &P);
    const long long n = P.g.n;
    const double* dx = x;
    double* dy = y;
    Buf bx, by;
    if (!P.device_inputs) {
      bx = Buf(sizeof(double) * n, ctx->stream);
      by = Buf(sizeof(double) * n, ctx->stream);
      PDEB_CUDA(cudaMemcpyAsync(bx.as<double>(), x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
      dx = bx.as<double>();
      dy = by.as<double>();
    }
    pdeb200_status s = apply_dev(ctx, P, dx, dy);
    if (!P.device_inputs)
      PDEB_CUDA(cudaMemcpyAsync(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
    return s;
  });
}

pdeb200_status pdeb200_time_series(const pdeb200_problem* prob, const pdeb200_time_options* topt,
                                   pdeb200_frame_cb on_frame, void* user, double* out_grid,
                                   pdeb200_report* report) {
  const double t0 = now_ms();
  if (report) std::memset(report, 0, sizeof(*report));
  if (!prob || !topt || !out_grid) return PDEB200_ERR_INVALID;
  pdeb200_status st = guarded(report, [&]() -> pdeb200_status {
    Context* ctx = get_context(topt->device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    return time_series_on(ctx, prob, topt, on_frame, user, out_grid, report);
  });
  if (report) report->total_ms = now_ms() - t0;
  return st;
}

pdeb200_status pdeb200_project_velocity(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                        double dt, double* u, double* v, double* w, double* pressure,
                                        const pdeb200_projection_options* popt,
                                        pdeb200_projection_report* report) {
  if (report) std::memset(report, 0, sizeof(*report));
  if (!u || !v || !pressure || !popt || (nz > 1 && !w) || nx < 2 || ny < 2 || dt == 0.0)
    return PDEB200_ERR_INVALID;
  pdeb200_report tmp{};
  pdeb200_status st = guarded(&tmp, [&]() -> pdeb200_status {
    Context* ctx = get_context(popt->device);
    std::lock_guard<std::mutex> lk(ctx->mu);
    return project_dev(ctx, nx, ny, nz, dx, dy, dz, dt, u, v, w, pressure, popt, report);
  });
  if (report && tmp.message[0]) std::memcpy(report->message, tmp.message, sizeof(report->message));
  return st;
}

}  // extern "C"
