// Serving loop of libpdeb200 (include/pdeb200_server.h): a request queue,
// admission against an HBM budget, and lanes (host thread + CUDA stream +
// solver context each) that pull admitted work and run it concurrently on the
// device. Mixed-precision Poisson requests that wait together are solved as
// one batched group (pdeb200_batch), so a lane turns every request admitted
// since its last group into one set of launches.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/pdeb200_server.h"
#include "host.h"

namespace pdeb {

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void face_dims_of(int f, int nx, int ny, int nz, int* w, int* h) {
  if (f <= kRight) {
    *w = ny;
    *h = nz;
  } else if (f <= kTop) {
    *w = nx;
    *h = nz;
  } else {
    *w = nx;
    *h = ny;
  }
}

}  // namespace

struct SReq {
  int64_t id = 0;
  int kind = 0;
  pdeb200_problem prob{};
  std::vector<double> f, k, nodal, u0;
  std::vector<double> fa[6][4];
  std::vector<pdeb200_nonlinear_term> nl;
  std::vector<double> pu, pv, pw, pp;
  int steps = 0;
  double tol = 1e-10, t_start = 0.0, dt = 0.0;
  int nx = 0, ny = 0, nz = 1, max_iter = 0;
  double dx = 0, dy = 0, dz = 0, pdt = 0, ptol = 0;
  double* out = nullptr;
  long long n = 0;
  int64_t bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  pdeb200_result res{};
  bool done = false;
};

struct Server {
  int dev = 0;
  int nlanes = 4;
  int max_batch = 64;
  int precision = PDEB200_MIXED;
  int queue_cap = 65536;
  int single_below = 0;
  int64_t budget = 0;
  pdeb200_batch_options bopt{};
  std::mutex mu;
  std::condition_variable cv;
  std::deque<SReq*> pending;
  std::unordered_map<int64_t, SReq*> reqs;
  int64_t next_id = 1;
  int64_t in_use = 0, peak = 0;
  int64_t submitted = 0, completed = 0, failed = 0, rejected = 0, running = 0;
  int busy = 0, busy_peak = 0;
  std::vector<double> lat;
  double t_reset = 0;
  bool stop = false;
  std::vector<std::thread> threads;
  std::vector<std::unique_ptr<Context>> ctxs;

  // Takes the next admissible work from the queue (caller holds mu). `single`
  // says that a mixed Poisson request is to be solved on its own grid: fewer
  // than single_below of them wait, so each free lane takes one.
  std::vector<SReq*> take(bool& single) {
    std::vector<SReq*> got;
    single = false;
    if (precision == PDEB200_MIXED && single_below > 1) {
      int waiting = 0;
      for (SReq* r : pending)
        if (r->kind == PDEB200_REQ_POISSON && ++waiting >= single_below) break;
      single = waiting < single_below;
    }
    for (auto it = pending.begin(); it != pending.end();) {
      SReq* r = *it;
      const bool batchable = r->kind == PDEB200_REQ_POISSON && precision == PDEB200_MIXED && !single;
      if (!got.empty()) {
        // a group holds mixed-precision Poisson requests of one tolerance
        if (!batchable || r->tol != got.front()->tol || (int)got.size() >= max_batch) {
          ++it;
          continue;
        }
      }
      if (in_use + r->bytes > budget) {
        ++it;
        continue;
      }
      in_use += r->bytes;
      peak = std::max(peak, in_use);
      got.push_back(r);
      it = pending.erase(it);
      if (!batchable) break;
    }
    return got;
  }

  void finish(SReq* r) {
    r->t_done = now_s();
    r->res.id = r->id;
    r->res.kind = r->kind;
    r->res.queue_ms = (r->t_admit - r->t_submit) * 1e3;
    r->res.run_ms = (r->t_done - r->t_admit) * 1e3;
    r->res.latency_ms = (r->t_done - r->t_submit) * 1e3;
    r->done = true;
    in_use -= r->bytes;
    --running;
    if (r->res.status == PDEB200_OK)
      ++completed;
    else
      ++failed;
    lat.push_back(r->res.latency_ms);
  }

  void run_group(Context* ctx, std::vector<SReq*>& g);
  void run_one(Context* ctx, SReq* r, bool mixed);
  void lane(int q);
};

static void set_msg(pdeb200_result* r, const char* m) {
  std::strncpy(r->message, m, sizeof(r->message) - 1);
  r->message[sizeof(r->message) - 1] = '\0';
}

void Server::run_group(Context* ctx, std::vector<SReq*>& g) {
  std::vector<pdeb200_problem> probs;
  for (auto* r : g) probs.push_back(r->prob);
  pdeb200_batch_options o = bopt;
  o.device = dev;
  o.stream = ctx->stream;
  o.autotune = 0;
  pdeb200_batch* b = nullptr;
  char msg[256];
  pdeb200_status st = pdeb200_batch_create(probs.data(), (int32_t)probs.size(), &o, &b, msg, sizeof(msg));
  if (st != PDEB200_OK) {
    for (auto* r : g) {
      r->res.status = st;
      set_msg(&r->res, msg);
    }
    return;
  }
  std::vector<pdeb200_report> reps(g.size());
  pdeb200_batch_solve(b, g.front()->tol, reps.data(), nullptr);
  for (size_t q = 0; q < g.size(); ++q) {
    SReq* r = g[q];
    // the result goes where the request's fields live (host or device)
    const pdeb200_status rs = pdeb200_batch_read_member(b, (int32_t)q, r->out, r->prob.mem_space);
    r->res.status = rs != PDEB200_OK ? rs : (reps[q].converged ? PDEB200_OK : PDEB200_ERR_NOT_CONVERGED);
    r->res.iterations = reps[q].iterations;
    r->res.rel_residual = reps[q].rel_residual;
    r->res.group_size = (int32_t)g.size();
    set_msg(&r->res, reps[q].message);
  }
  pdeb200_batch_destroy(b);
}

void Server::run_one(Context* ctx, SReq* r, bool mixed) {
  r->res.group_size = 1;
  try {
    if (r->kind == PDEB200_REQ_POISSON) {
      pdeb200_options o;
      pdeb200_default_options(&o);
      o.method = PDEB200_MG_PCG;
      if (mixed) o.precision = PDEB200_MIXED;
      o.tol = r->tol;
      o.tol_mode = PDEB200_TOL_RELATIVE;
      o.max_iter = 500;
      o.device = dev;
      pdeb200_report rep{};
      r->res.status = solve_on(ctx, &r->prob, &o, r->out, &rep);
      r->res.iterations = rep.iterations;
      r->res.rel_residual = rep.rel_residual;
      set_msg(&r->res, rep.message);
    } else if (r->kind == PDEB200_REQ_HEAT) {
      pdeb200_time_options t{};
      t.t_start = r->t_start;
      t.dt = r->dt;
      t.frames = r->steps + 1;  // frame 0 is u0; each further frame is one step
      t.frame_stride = r->steps > 0 ? r->steps : 1;
      t.device = dev;
      pdeb200_report rep{};
      r->res.status = time_series_on(ctx, &r->prob, &t, nullptr, nullptr, r->out, &rep);
      r->res.iterations = r->steps;
      set_msg(&r->res, rep.message);
    } else {
      pdeb200_projection_options po{};
      po.max_iter = r->max_iter > 0 ? r->max_iter : 10000;
      po.tol = r->ptol > 0 ? r->ptol : 1e-10;
      po.device = dev;
      po.mem_space = PDEB200_MEM_HOST;
      po.fix_pressure_corner = 1;
      pdeb200_projection_report rep{};
      const bool is3 = r->nz > 1;
      r->res.status = project_dev(ctx, r->nx, r->ny, r->nz, r->dx, r->dy, r->dz, r->pdt, r->pu.data(), r->pv.data(),
                                  is3 ? r->pw.data() : nullptr, r->pp.data(), &po, &rep);
      PDEB_CUDA(cudaStreamSynchronize(ctx->stream));
      const size_t n = (size_t)r->n;
      double* o = r->out;
      std::memcpy(o, r->pu.data(), sizeof(double) * n);
      std::memcpy(o + n, r->pv.data(), sizeof(double) * n);
      size_t at = 2 * n;
      if (is3) {
        std::memcpy(o + at, r->pw.data(), sizeof(double) * n);
        at += n;
      }
      std::memcpy(o + at, r->pp.data(), sizeof(double) * n);
      r->res.iterations = rep.poisson_iterations;
      r->res.rel_residual = rep.poisson_residual;
      set_msg(&r->res, rep.message);
    }
  } catch (const StatusFailure& s) {
    r->res.status = s.status;
    set_msg(&r->res, s.what.c_str());
  } catch (const CudaFailure& c) {
    cudaGetLastError();
    r->res.status = PDEB200_ERR_CUDA;
    set_msg(&r->res, c.what.c_str());
  }
}

void Server::lane(int q) {
  cudaSetDevice(dev);
  Context* ctx = ctxs[q].get();
  for (;;) {
    std::vector<SReq*> work;
    bool single = false;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] {
        if (stop) return true;
        work = take(single);
        return !work.empty();
      });
      if (stop && work.empty()) return;
      const double t = now_s();
      for (auto* r : work) {
        r->t_admit = t;
        ++running;
      }
      ++busy;
      busy_peak = std::max(busy_peak, busy);
    }
    const bool mixed_poisson = work.front()->kind == PDEB200_REQ_POISSON && precision == PDEB200_MIXED;
    if (mixed_poisson && !single)
      run_group(ctx, work);
    else
      run_one(ctx, work.front(), mixed_poisson);
    {
      std::lock_guard<std::mutex> lk(mu);
      for (auto* r : work) finish(r);
      --busy;
    }
    cv.notify_all();
  }
}

static int64_t estimate_bytes(const SReq& r, int precision) {
  const int64_t n = r.n;
  switch (r.kind) {
    case PDEB200_REQ_POISSON:
      return (precision == PDEB200_MIXED ? 80 : 128) * n + (1 << 20);
    case PDEB200_REQ_HEAT:
      return 64 * n + (1 << 20);
    default:
      return 96 * n + (1 << 20);
  }
}

static void copy_problem(SReq* r, const pdeb200_problem* p) {
  r->prob = *p;
  const int nz = p->nz > 1 ? p->nz : 1;
  r->n = (long long)p->nx * p->ny * nz;
  const size_t n = (size_t)r->n;
  auto grab = [&](const double* src, size_t cnt, std::vector<double>* dst) -> const double* {
    if (!src) return nullptr;
    dst->assign(src, src + cnt);
    return dst->data();
  };
  // device-resident fields are used in place (the caller keeps them until the
  // request completes); host fields are copied
  const bool dev = p->mem_space == PDEB200_MEM_DEVICE;
  r->prob.f = dev ? p->f : grab(p->f, n, &r->f);
  r->prob.k = dev ? p->k : grab(p->k, n, &r->k);
  r->prob.nodal = dev ? p->nodal : grab(p->nodal, 7 * n, &r->nodal);
  r->prob.u0 = dev ? p->u0 : grab(p->u0, n, &r->u0);
  for (int f = 0; f < 6; ++f) {
    int w, h;
    face_dims_of(f, p->nx, p->ny, nz, &w, &h);
    const size_t cnt = (size_t)w * h;
    r->prob.face[f].value_arr = grab(p->face[f].value_arr, cnt, &r->fa[f][0]);
    r->prob.face[f].alpha_arr = grab(p->face[f].alpha_arr, cnt, &r->fa[f][1]);
    r->prob.face[f].beta_arr = grab(p->face[f].beta_arr, cnt, &r->fa[f][2]);
    r->prob.face[f].gamma_arr = grab(p->face[f].gamma_arr, cnt, &r->fa[f][3]);
  }
  // nonlinear terms are a host array in every memory space: copied
  if (p->n_nonlinear > 0 && p->nonlinear) {
    r->nl.assign(p->nonlinear, p->nonlinear + p->n_nonlinear);
    r->prob.nonlinear = r->nl.data();
  } else {
    r->prob.n_nonlinear = 0;
    r->prob.nonlinear = nullptr;
  }
}

}  // namespace pdeb

struct pdeb200_server {
  pdeb::Server s;
};

extern "C" {

pdeb200_status pdeb200_server_create(const pdeb200_server_options* opt, pdeb200_server** out, char* message,
                                     size_t message_len) {
  using namespace pdeb;
  auto msg = [&](const std::string& m) {
    if (message && message_len) {
      std::strncpy(message, m.c_str(), message_len - 1);
      message[message_len - 1] = '\0';
    }
  };
  msg("");
  if (!opt || !out) return PDEB200_ERR_INVALID;
  *out = nullptr;
  pdeb200_server* h = nullptr;
  try {
    get_context(opt->device);
    h = new pdeb200_server();
    Server& S = h->s;
    S.dev = opt->device;
    S.nlanes = opt->lanes > 0 ? opt->lanes : 4;
    S.max_batch = opt->max_batch > 0 ? opt->max_batch : 64;
    S.precision = opt->precision == PDEB200_FP64 ? PDEB200_FP64 : PDEB200_MIXED;
    S.queue_cap = opt->queue_capacity > 0 ? opt->queue_capacity : 65536;
    S.single_below = opt->single_below;
    S.bopt = opt->batch;
    size_t fr = 0, tot = 0;
    PDEB_CUDA(cudaMemGetInfo(&fr, &tot));
    S.budget = opt->hbm_budget_bytes > 0 ? opt->hbm_budget_bytes : (int64_t)(0.8 * (double)fr);
    S.t_reset = now_s();
    for (int q = 0; q < S.nlanes; ++q) {
      S.ctxs.emplace_back(new Context());
      init_context(S.ctxs.back().get(), S.dev);
    }
    for (int q = 0; q < S.nlanes; ++q) S.threads.emplace_back([&S, q] { S.lane(q); });
    *out = h;
    return PDEB200_OK;
  } catch (const StatusFailure& s) {
    msg(s.what);
    delete h;
    return s.status;
  } catch (const CudaFailure& c) {
    msg(c.what);
    cudaGetLastError();
    delete h;
    return PDEB200_ERR_CUDA;
  }
}

pdeb200_status pdeb200_server_submit(pdeb200_server* h, const pdeb200_request* req, int64_t* id) {
  using namespace pdeb;
  if (!h || !req || !req->out) return PDEB200_ERR_INVALID;
  Server& S = h->s;
  auto r = std::make_unique<SReq>();
  r->kind = req->kind;
  r->out = req->out;
  if (req->kind == PDEB200_REQ_POISSON || req->kind == PDEB200_REQ_HEAT) {
    if (!req->problem) return PDEB200_ERR_INVALID;
    copy_problem(r.get(), req->problem);
    r->tol = req->tol > 0 ? req->tol : 1e-10;
    r->steps = req->steps;
    r->t_start = req->t_start;
    r->dt = req->dt;
    if (req->kind == PDEB200_REQ_HEAT && (req->steps <= 0 || req->dt <= 0.0)) return PDEB200_ERR_INVALID;
  } else if (req->kind == PDEB200_REQ_PROJECTION) {
    const bool is3 = req->nz > 1;
    if (!req->u || !req->v || !req->p || (is3 && !req->w) || req->nx < 2 || req->ny < 2 || req->proj_dt == 0.0)
      return PDEB200_ERR_INVALID;
    r->nx = req->nx;
    r->ny = req->ny;
    r->nz = is3 ? req->nz : 1;
    r->n = (long long)r->nx * r->ny * r->nz;
    r->dx = req->dx;
    r->dy = req->dy;
    r->dz = req->dz;
    r->pdt = req->proj_dt;
    r->ptol = req->proj_tol;
    r->max_iter = req->max_iter;
    r->pu.assign(req->u, req->u + r->n);
    r->pv.assign(req->v, req->v + r->n);
    if (is3) r->pw.assign(req->w, req->w + r->n);
    r->pp.assign(req->p, req->p + r->n);
  } else {
    return PDEB200_ERR_INVALID;
  }
  // a mixed request that may run on its own grid is admitted at the FP64
  // path's estimate, which bounds the single-grid mixed working set
  r->bytes = estimate_bytes(*r, S.precision == PDEB200_MIXED && S.single_below > 1 ? PDEB200_FP64 : S.precision);
  std::lock_guard<std::mutex> lk(S.mu);
  if (r->bytes > S.budget) {
    ++S.rejected;
    return PDEB200_ERR_OOM;
  }
  if ((int)S.pending.size() >= S.queue_cap) {
    ++S.rejected;
    return PDEB200_ERR_BUSY;
  }
  r->id = S.next_id++;
  r->t_submit = now_s();
  if (id) *id = r->id;
  SReq* raw = r.release();
  S.reqs[raw->id] = raw;
  S.pending.push_back(raw);
  ++S.submitted;
  S.cv.notify_all();
  return PDEB200_OK;
}

pdeb200_status pdeb200_server_wait(pdeb200_server* h, int64_t id, double timeout_ms, pdeb200_result* res) {
  using namespace pdeb;
  if (!h) return PDEB200_ERR_INVALID;
  Server& S = h->s;
  std::unique_lock<std::mutex> lk(S.mu);
  auto it = S.reqs.find(id);
  if (it == S.reqs.end()) return PDEB200_ERR_INVALID;
  SReq* r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_ms < 0)
    S.cv.wait(lk, ready);
  else if (!S.cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready))
    return PDEB200_ERR_TIMEOUT;
  if (res) *res = r->res;
  const pdeb200_status st = (pdeb200_status)r->res.status;
  S.reqs.erase(it);
  delete r;
  return st;
}

pdeb200_status pdeb200_server_drain(pdeb200_server* h, double timeout_ms) {
  using namespace pdeb;
  if (!h) return PDEB200_ERR_INVALID;
  Server& S = h->s;
  std::unique_lock<std::mutex> lk(S.mu);
  auto idle = [&] { return S.pending.empty() && S.running == 0; };
  if (timeout_ms < 0)
    S.cv.wait(lk, idle);
  else if (!S.cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), idle))
    return PDEB200_ERR_TIMEOUT;
  return PDEB200_OK;
}

pdeb200_status pdeb200_server_get_stats(pdeb200_server* h, pdeb200_server_stats* st, int32_t reset) {
  using namespace pdeb;
  if (!h || !st) return PDEB200_ERR_INVALID;
  Server& S = h->s;
  std::lock_guard<std::mutex> lk(S.mu);
  std::memset(st, 0, sizeof(*st));
  st->submitted = S.submitted;
  st->completed = S.completed;
  st->failed = S.failed;
  st->rejected = S.rejected;
  st->in_flight = S.running;
  st->queued = (int64_t)S.pending.size();
  st->bytes_in_use = S.in_use;
  st->bytes_peak = S.peak;
  st->budget_bytes = S.budget;
  st->lanes_busy_peak = S.busy_peak;
  std::vector<double> l = S.lat;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
      const double pos = p * (double)(l.size() - 1);
      const size_t a = (size_t)pos;
      const size_t b = std::min(a + 1, l.size() - 1);
      return l[a] + (pos - (double)a) * (l[b] - l[a]);
    };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = l.back();
  }
  st->elapsed_s = now_s() - S.t_reset;
  st->solves_per_s = st->elapsed_s > 0 ? (double)l.size() / st->elapsed_s : 0.0;
  if (reset) {
    S.lat.clear();
    S.t_reset = now_s();
    S.busy_peak = S.busy;
    S.peak = S.in_use;
  }
  return PDEB200_OK;
}

void pdeb200_server_destroy(pdeb200_server* h) {
  using namespace pdeb;
  if (!h) return;
  Server& S = h->s;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    S.stop = true;
  }
  S.cv.notify_all();
  for (auto& t : S.threads) t.join();
  for (auto& c : S.ctxs) free_context(c.get());
  for (auto& kv : S.reqs) delete kv.second;
  delete h;
}

}  // extern "C"
