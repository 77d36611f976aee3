// Batched solver host side: plan construction (members, hierarchies, packed
// device arenas), tile tables, the refinement cycle as a CUDA graph, lazy
// polling, the autotuner with its on-disk cache, and the pdeb200_batch_* C ABI.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pdeb200_batch.h"
#include "batch_kernels.cuh"
#include "host.h"
#include "solvers.cuh"

namespace pdeb {

struct BatchParams {
  int tile_x = 32, tile_y = 16, tile_z = 8;
  int pre = 2, post = 2, coarse_sweeps = 16;
  int max_inner = 40, max_outer = 12;
  double inner_tol = 1e-4;
};

struct Sched;

struct BatchPlan {
  int dev = 0;
  Context cx;  // carries the stream for the shared upload helpers
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool bf16 = false;
  bool use_graph = true;
  int count = 0;
  int lmax = 0;
  BatchParams prm;
  std::vector<DevProblem> probs;
  std::vector<BLevel> levels;      // host copy of the level records
  std::vector<int> lev0;           // member -> level-0 record
  std::vector<int> nlev;           // member -> number of levels
  std::vector<long long> off;      // member -> offset in the packed arrays
  std::vector<BMember> mem_tmpl;   // member records without solve state
  long long nodes = 0;
  Buf a64, a32, akh;               // packed arenas
  double *f64 = nullptr, *b64 = nullptr, *x64 = nullptr;
  std::vector<Buf> owned;          // face arrays of coarse levels
  Buf d_levels, d_mem, d_active;
  std::unique_ptr<Sched> full;  // tiles of every member (set by build_schedule)
  int* h_active = nullptr;
  BMember* h_mem = nullptr;
  bool compact = true;  // rebuild the tables for the unfinished members as they thin out
  int last_compactions = 0;
  long long last_launches = 0;
  int last_cycles = 0;
  double last_ms = 0.0, tune_ms = 0.0;
  bool tuned_from_cache = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  ~BatchPlan();
};

// Tile tables of one schedule (all members, or the unfinished ones), the
// reduction partials sized for its level-0 tiles, each member's level-0 tile
// range and the captured cycle.
struct Sched {
  Buf tiles, partials;
  std::vector<long long> off, cnt;
  std::vector<int> tile0, ntiles;  // per member; ntiles 0 when absent
  int lmax = 0;
  int members = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;
  Sched() = default;
  Sched(const Sched&) = delete;
  Sched& operator=(const Sched&) = delete;
  ~Sched() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

BatchPlan::~BatchPlan() {
  {
    if (stream) cudaStreamSynchronize(stream);
    full.reset();
    if (h_active) cudaFreeHost(h_active);
    if (h_mem) cudaFreeHost(h_mem);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    owned.clear();
    probs.clear();
    a64.reset();
    a32.reset();
    akh.reset();
    d_levels.reset();
    d_mem.reset();
    d_active.reset();
    if (stream) cudaStreamSynchronize(stream);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }
}

namespace {

constexpr long long kAlign = 64;  // elements per array slot (>= 256 B for FP32 and FP64)

long long pad(long long n) { return (n + kAlign - 1) / kAlign * kAlign; }

long long interior_nodes(const GridDev& g) {
  return (long long)(g.nx - 2) * (g.ny - 2) * (g.dim == 3 ? g.nz - 2 : 1);
}

// Tiles of one level of one member (interior nodes only).
void make_tiles(const GridDev& g, bool coarse, const BatchParams& p, int lev, int member, std::vector<BTile>* out) {
  const int ni = g.nx - 2, nj = g.ny - 2;
  const int kb = g.dim == 3 ? 1 : 0, ke = g.dim == 3 ? g.nz - 1 : 1;
  auto tile = [&](int x0, int y0, int w, int h, int z0, int z1, int coarse_flag) {
    if (w > 65535 || h > 65535) throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "coarsest level too wide for one tile"};
    BTile t{};
    t.lev = lev;
    t.member = member;
    t.x0 = x0;
    t.y0 = y0;
    t.z0 = z0;
    t.z1 = z1;
    t.w = (unsigned short)w;
    t.h = (unsigned short)h;
    int lw = 0;
    while ((1 << lw) < w) ++lw;
    t.lw = (unsigned char)lw;
    t.coarse = (unsigned char)coarse_flag;
    out->push_back(t);
  };
  if (coarse) {
    tile(0, 0, ni, nj, kb, ke, 1);
    return;
  }
  const int tw = g.dim == 3 ? 32 : p.tile_x;
  const int th = g.dim == 3 ? 8 : p.tile_y;
  const int tz = g.dim == 3 ? p.tile_z : 1;
  for (int z = kb; z < ke; z += tz)
    for (int y = 0; y < nj; y += th)
      for (int x = 0; x < ni; x += tw) {
        // regular tiles keep the full row width so a warp stays on one row
        tile(x, y, std::min(tw, ni - x), std::min(th, nj - y), z, std::min(ke, z + tz), 0);
        out->back().lw = (unsigned char)(tw == 64 ? 6 : 5);
      }
}

template <typename KT>
void enqueue_cycle(BatchPlan& B, Sched& Sc) {
  const BTile* tiles = Sc.tiles.as<BTile>();
  const BLevel* lv = B.d_levels.as<BLevel>();
  BMember* mem = B.d_mem.as<BMember>();
  double* part = Sc.partials.as<double>();
  int* active = B.d_active.as<int>();
  cudaStream_t s = B.stream;
  const int T = kBThreads;
  auto S = [&](int l) { return tiles + Sc.off[l]; };
  auto N = [&](int l) { return (unsigned)Sc.cnt[l]; };
  long long launches = 0;
  kb_xupdate<<<N(0), T, 0, s>>>(S(0), lv, mem);
  kb_outer<<<N(0), T, 0, s>>>(S(0), lv, mem, part, active);
  kb_apply_pq<<<N(0), T, 0, s>>>(S(0), lv, mem, part);
  kb_update<<<N(0), T, 0, s>>>(S(0), lv, mem, part);
  launches += 4;
  for (int l = 0; l + 1 < Sc.lmax; ++l) {
    for (int q = 0; q < B.prm.pre; ++q) {
      kb_smooth<KT><<<N(l), T, 0, s>>>(S(l), lv, mem, 0, q == 0 ? 1 : 0);
      kb_smooth<KT><<<N(l), T, 0, s>>>(S(l), lv, mem, 1, 0);
      launches += 2;
    }
    kb_residual<KT><<<N(l), T, 0, s>>>(S(l), lv, mem);
    kb_restrict<KT><<<N(l + 1), T, 0, s>>>(S(l + 1), lv, mem, B.prm.coarse_sweeps);
    launches += 2;
  }
  for (int l = Sc.lmax - 2; l >= 0; --l) {
    kb_prolong<<<N(l), T, 0, s>>>(S(l), lv, mem);
    ++launches;
    for (int q = 0; q < B.prm.post; ++q) {
      kb_smooth<KT><<<N(l), T, 0, s>>>(S(l), lv, mem, 1, 0);
      kb_smooth<KT><<<N(l), T, 0, s>>>(S(l), lv, mem, 0, 0);
      launches += 2;
    }
  }
  kb_rz<<<N(0), T, 0, s>>>(S(0), lv, mem, part);
  kb_pupdate<<<N(0), T, 0, s>>>(S(0), lv, mem);
  launches += 2;
  Sc.launches = launches;
  PDEB_CUDA(cudaGetLastError());
}

void run_cycle_enqueue(BatchPlan& B, Sched& Sc) {
  if (B.bf16)
    enqueue_cycle<__nv_bfloat16>(B, Sc);
  else
    enqueue_cycle<float>(B, Sc);
}

// Tile tables of `subset` (every member when null), member tile ranges and the
// captured cycle for the current parameters.
std::unique_ptr<Sched> make_sched(BatchPlan& B, const std::vector<int>* subset) {
  auto Sc = std::make_unique<Sched>();
  std::vector<int> all_m;
  if (!subset) {
    all_m.resize(B.count);
    for (int m = 0; m < B.count; ++m) all_m[m] = m;
    subset = &all_m;
  }
  Sc->members = (int)subset->size();
  for (int m : *subset) Sc->lmax = std::max(Sc->lmax, B.nlev[m]);
  Sc->tile0.assign(B.count, 0);
  Sc->ntiles.assign(B.count, 0);
  std::vector<std::vector<BTile>> per(Sc->lmax);
  for (int m : *subset) {
    for (int l = 0; l < B.nlev[m]; ++l) {
      const int rec = B.lev0[m] + l;
      const BLevel& L = B.levels[rec];
      if (l == 0) Sc->tile0[m] = (int)per[0].size();
      make_tiles(L.g, L.coarsest != 0, B.prm, rec, m, &per[l]);
      if (l == 0) Sc->ntiles[m] = (int)per[0].size() - Sc->tile0[m];
    }
  }
  std::vector<BTile> all;
  Sc->off.assign(Sc->lmax, 0);
  Sc->cnt.assign(Sc->lmax, 0);
  for (int l = 0; l < Sc->lmax; ++l) {
    Sc->off[l] = (long long)all.size();
    Sc->cnt[l] = (long long)per[l].size();
    all.insert(all.end(), per[l].begin(), per[l].end());
  }
  if (Sc->cnt[0] >= (1LL << 31)) throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "batch has too many tiles"};
  Sc->tiles = Buf(sizeof(BTile) * all.size(), B.stream);
  PDEB_CUDA(cudaMemcpyAsync(Sc->tiles.as<void>(), all.data(), sizeof(BTile) * all.size(), cudaMemcpyHostToDevice,
                            B.stream));
  Sc->partials = Buf(sizeof(double) * (size_t)Sc->cnt[0], B.stream);
  PDEB_CUDA(cudaStreamSynchronize(B.stream));
  if (B.use_graph) {
    PDEB_CUDA(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
    try {
      run_cycle_enqueue(B, *Sc);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(B.stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    PDEB_CUDA(cudaStreamEndCapture(B.stream, &Sc->graph));
    PDEB_CUDA(cudaGraphInstantiate(&Sc->exec, Sc->graph, 0));
  }
  return Sc;
}

void build_schedule(BatchPlan& B) {
  B.full.reset();
  B.full = make_sched(B, nullptr);
  for (int m = 0; m < B.count; ++m) {
    B.mem_tmpl[m].tile0 = B.full->tile0[m];
    B.mem_tmpl[m].ntiles = B.full->ntiles[m];
  }
}

// One solve of every member; returns the number of unconverged members.
int solve_all(BatchPlan& B, double tol, int max_cycles_cap = 0) {
  // member records: fresh solve state
  for (int m = 0; m < B.count; ++m) {
    BMember& M = B.h_mem[m];
    M = B.mem_tmpl[m];
    M.state = kBNeedOuter;
    M.outer = M.inner = M.inner_total = 0;
    M.first = 0;
    M.status = PDEB200_ERR_NOT_CONVERGED;
    M.e_valid = 0;
    M.ticket = 0u;
    M.bb = M.rr0 = M.rr = M.rr_outer = M.rz = M.alpha = M.beta = 0.0;
    M.tol2 = tol * tol;
    M.tol2_inner = B.prm.inner_tol * B.prm.inner_tol;
    M.tol2_step = M.tol2_inner;
    M.max_inner = B.prm.max_inner;
    M.max_outer = B.prm.max_outer;
  }
  *B.h_active = B.count;
  PDEB_CUDA(cudaEventRecord(B.ev0, B.stream));
  PDEB_CUDA(cudaMemcpyAsync(B.d_mem.as<void>(), B.h_mem, sizeof(BMember) * B.count, cudaMemcpyHostToDevice,
                            B.stream));
  PDEB_CUDA(cudaMemcpyAsync(B.d_active.as<void>(), B.h_active, sizeof(int), cudaMemcpyHostToDevice, B.stream));
  const BLevel* lv = B.d_levels.as<BLevel>();
  kb_rhs<<<(unsigned)B.full->cnt[0], kBThreads, 0, B.stream>>>(B.full->tiles.as<BTile>(), lv,
                                                               B.d_mem.as<BMember>());
  long long launches = 1;
  const int max_cycles =
      max_cycles_cap > 0 ? max_cycles_cap : B.prm.max_outer * (B.prm.max_inner + 2) + 8;
  Sched* cur = B.full.get();
  std::unique_ptr<Sched> part;  // tables of the unfinished members, once they thin out
  int compactions = 0;
  int cycles = 0, batch = 2, prev_active = B.count;
  while (cycles < max_cycles) {
    const int nb = std::min(batch, max_cycles - cycles);
    for (int q = 0; q < nb; ++q) {
      if (cur->exec) {
        PDEB_CUDA(cudaGraphLaunch(cur->exec, B.stream));
      } else {
        run_cycle_enqueue(B, *cur);
      }
      launches += cur->launches;
    }
    cycles += nb;
    PDEB_CUDA(cudaMemcpyAsync(B.h_active, B.d_active.as<void>(), sizeof(int), cudaMemcpyDeviceToHost, B.stream));
    PDEB_CUDA(cudaStreamSynchronize(B.stream));
    if (*B.h_active <= 0) break;
    // poll often once members finish (compaction follows them), rarely before
    batch = *B.h_active < prev_active ? 2 : std::min(batch * 2, 8);
    prev_active = *B.h_active;
    // Compaction: when at most half the members in the tables are unfinished,
    // rebuild the tables (and the captured cycle) for those alone. A member's
    // tiles and their order do not change, so neither do its numbers.
    if (B.compact && *B.h_active * 2 <= cur->members && compactions < 4) {
      PDEB_CUDA(cudaMemcpyAsync(B.h_mem, B.d_mem.as<void>(), sizeof(BMember) * B.count, cudaMemcpyDeviceToHost,
                                B.stream));
      PDEB_CUDA(cudaStreamSynchronize(B.stream));
      std::vector<int> act;
      for (int m = 0; m < B.count; ++m)
        if (B.h_mem[m].state != kBDone) act.push_back(m);
      std::unique_ptr<Sched> next = make_sched(B, &act);
      for (int m : act) {
        B.h_mem[m].tile0 = next->tile0[m];
        B.h_mem[m].ntiles = next->ntiles[m];
      }
      PDEB_CUDA(cudaMemcpyAsync(B.d_mem.as<void>(), B.h_mem, sizeof(BMember) * B.count, cudaMemcpyHostToDevice,
                                B.stream));
      part = std::move(next);
      cur = part.get();
      ++compactions;
    }
  }
  B.last_compactions = compactions;
  kb_fill_boundary<<<B.count, kBThreads, 0, B.stream>>>(lv, B.d_mem.as<BMember>());
  ++launches;
  PDEB_CUDA(cudaGetLastError());
  PDEB_CUDA(cudaEventRecord(B.ev1, B.stream));
  PDEB_CUDA(cudaMemcpyAsync(B.h_mem, B.d_mem.as<void>(), sizeof(BMember) * B.count, cudaMemcpyDeviceToHost,
                            B.stream));
  PDEB_CUDA(cudaStreamSynchronize(B.stream));
  float ms = 0.f;
  PDEB_CUDA(cudaEventElapsedTime(&ms, B.ev0, B.ev1));
  B.last_ms = ms;
  B.last_cycles = cycles;
  B.last_launches = launches;
  int open = 0;
  for (int m = 0; m < B.count; ++m)
    if (B.h_mem[m].status != PDEB200_OK) ++open;
  return open;
}

// ------------------------------------------------------------ construction

// Coarse hierarchy k of every member at level depth d, in one launch: block q
// fills level record recs[q] from its finer record by nearest-node injection.
template <typename KT>
__global__ void kb_inject(const int* __restrict__ recs, const BLevel* __restrict__ lv) {
  const BLevel& C = lv[recs[blockIdx.x]];
  const BLevel& F = lv[C.prev];
  const KT* kf = static_cast<const KT*>(F.kh);
  KT* kc = static_cast<KT*>(const_cast<void*>(C.kh));
  const GridDev& gc = C.g;
  const GridDev& gf = F.g;
  for (long long t = threadIdx.x; t < gc.n; t += blockDim.x) {
    const int I = int(t % gc.nx);
    const int J = int((t / gc.nx) % gc.ny);
    const int K = int(t / gc.sxy);
    const int fi = nearest_fine(I, gf.nx, gc.nx), fj = nearest_fine(J, gf.ny, gc.ny);
    const int fk = gc.dim == 3 ? nearest_fine(K, gf.nz, gc.nz) : 0;
    kc[t] = kf[((long long)fk * gf.ny + fj) * gf.nx + fi];
  }
}

template <typename KT>
void fill_hierarchy_k(BatchPlan& B, KT* kh0, float* k32, const double* k64) {
  const long long n = B.nodes;
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
  k_convert<KT, double><<<blocks, 256, 0, B.stream>>>(n, kh0, k64);
  k_convert<float, double><<<blocks, 256, 0, B.stream>>>(n, k32, k64);
  std::vector<std::vector<int>> by_depth(B.lmax);
  for (size_t r = 0; r < B.levels.size(); ++r)
    if (B.levels[r].level > 0 && B.levels[r].kind == kDivk) by_depth[B.levels[r].level].push_back((int)r);
  std::vector<int> flat;
  std::vector<size_t> start(B.lmax, 0);
  for (int d = 1; d < B.lmax; ++d) {
    start[d] = flat.size();
    flat.insert(flat.end(), by_depth[d].begin(), by_depth[d].end());
  }
  if (flat.empty()) return;
  Buf recs(sizeof(int) * flat.size(), B.stream);
  PDEB_CUDA(cudaMemcpyAsync(recs.as<void>(), flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice,
                            B.stream));
  for (int d = 1; d < B.lmax; ++d)
    if (!by_depth[d].empty())
      kb_inject<KT><<<(unsigned)by_depth[d].size(), 256, 0, B.stream>>>(recs.as<int>() + start[d],
                                                                           B.d_levels.as<BLevel>());
  PDEB_CUDA(cudaGetLastError());
  PDEB_CUDA(cudaStreamSynchronize(B.stream));  // recs is released on return
}

void create_plan(BatchPlan& B, const pdeb200_problem* probs, int count, const pdeb200_batch_options* o) {
  if (!probs || count <= 0) throw StatusFailure{PDEB200_ERR_INVALID, "empty batch"};
  B.count = count;
  B.bf16 = o->bf16_coefficients != 0;
  B.use_graph = o->no_graph == 0;
  B.compact = o->no_compact == 0;
  B.dev = o->device;
  get_context(o->device);
  if (o->stream) {
    B.stream = static_cast<cudaStream_t>(o->stream);
  } else {
    PDEB_CUDA(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
    B.own_stream = true;
  }
  B.cx.dev = o->device;
  B.cx.stream = B.stream;
  B.cx.own_stream = nullptr;
  PDEB_CUDA(cudaEventCreate(&B.ev0));
  PDEB_CUDA(cudaEventCreate(&B.ev1));
  PDEB_CUDA(cudaMallocHost(&B.h_active, sizeof(int)));
  PDEB_CUDA(cudaMallocHost(&B.h_mem, sizeof(BMember) * count));

  // members: validation, geometry and faces of every level (host side)
  B.probs.resize(count);
  B.lev0.resize(count);
  B.nlev.resize(count);
  B.off.resize(count);
  B.mem_tmpl.assign(count, BMember{});
  long long n32 = 0, nkh = 0;
  std::vector<long long> x_off, b_off, r_off, kh_off;  // per level record (kh: levels >= 1 only)
  std::vector<long long> p_off(count), q_off(count), e_off(count);
  for (int m = 0; m < count; ++m) {
    const pdeb200_problem& hp = probs[m];
    if (hp.coef_kind != PDEB200_COEF_CONST && hp.coef_kind != PDEB200_COEF_DIVK)
      throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "batch members take COEF_CONST or COEF_DIVK"};
    if (hp.n_nonlinear > 0) throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "Multigrid requires linear PDEs"};
    describe_problem(&B.cx, &hp, &B.probs[m]);
    DevProblem& P = B.probs[m];
    B.off[m] = B.nodes;
    B.nodes += P.g.n;
    B.lev0[m] = (int)B.levels.size();
    BLevel L0{};
    L0.g = P.g;
    L0.kind = P.coef_kind == kDivk ? kDivk : kConst;
    L0.member = m;
    L0.prev = -1;
    L0.next = -1;
    L0.level = 0;
    L0.cc = P.cc;
    L0.ihx2 = P.cd.ihx2;
    L0.ihy2 = P.cd.ihy2;
    L0.ihz2 = P.cd.ihz2;
    L0.cx = P.cd.cx;
    L0.dyc = P.cd.dyc;
    L0.dzc = P.cd.dzc;
    L0.e = P.e;
    B.levels.push_back(L0);
    int nc[3];
    while (coarse_dims(B.levels.back().g, &hp, nc)) {
      const BLevel& F = B.levels.back();
      BLevel C = F;
      C.g.nx = nc[0];
      C.g.ny = nc[1];
      C.g.nz = F.g.dim == 3 ? nc[2] : 1;
      C.g.sxy = (long long)C.g.nx * C.g.ny;
      C.g.n = C.g.sxy * C.g.nz;
      const double cdx = (hp.xmax - hp.xmin) / (double)(C.g.nx - 1);
      const double cdy = (hp.ymax - hp.ymin) / (double)(C.g.ny - 1);
      const double cdz = C.g.dim == 3 ? (hp.zmax - hp.zmin) / (double)(C.g.nz - 1) : 0.0;
      build_faces(&B.cx, &hp, C.g.nx, C.g.ny, C.g.nz, cdx, cdy, cdz, 2, &C.g, &B.owned);
      if (C.kind == kConst) {
        C.cc = coarsen_coef(nullptr, P, P.cc, F.g, C.g, cdx, cdy, cdz, nullptr);
      } else {
        C.ihx2 = 1.0 / (cdx * cdx);
        C.ihy2 = 1.0 / (cdy * cdy);
        C.ihz2 = C.g.dim == 3 ? 1.0 / (cdz * cdz) : 0.0;
        C.cx = P.c / (2.0 * cdx);
        C.dyc = P.d / (2.0 * cdy);
        C.dzc = C.g.dim == 3 ? P.dzc / (2.0 * cdz) : 0.0;
      }
      C.prev = (int)B.levels.size() - 1;
      C.level = F.level + 1;
      B.levels.back().next = (int)B.levels.size();
      B.levels.push_back(C);
    }
    B.nlev[m] = (int)B.levels.size() - B.lev0[m];
    if (B.nlev[m] < 2)
      throw StatusFailure{PDEB200_ERR_UNSUPPORTED, "batch member too small for multigrid (needs a side of 5+ nodes)"};
    B.levels.back().coarsest = 1;
    B.lmax = std::max(B.lmax, B.nlev[m]);
    for (int l = 0; l < B.nlev[m]; ++l) {
      const long long n = B.levels[B.lev0[m] + l].g.n;
      x_off.push_back(n32);
      n32 += pad(n);
      b_off.push_back(n32);
      n32 += pad(n);
      r_off.push_back(n32);
      n32 += pad(n);
      if (l > 0 && P.coef_kind == kDivk) {
        kh_off.push_back(nkh);
        nkh += pad(n);
      } else {
        kh_off.push_back(-1);
      }
    }
    const long long n0 = pad(P.g.n);
    p_off[m] = n32;
    n32 += n0;
    q_off[m] = n32;
    n32 += n0;
    e_off[m] = n32;
    n32 += n0;
  }
  // arenas. FP64: f | b | x | k (packed in member order); FP32: k (packed),
  // level vectors and p, q, e; hierarchy k: level 0 packed, then coarse levels.
  const long long N = B.nodes;
  B.a64 = Buf(sizeof(double) * 4 * (size_t)N, B.stream);
  B.f64 = B.a64.as<double>();
  B.b64 = B.f64 + N;
  B.x64 = B.b64 + N;
  double* k64 = B.x64 + N;
  PDEB_CUDA(cudaMemsetAsync(B.a64.as<void>(), 0, sizeof(double) * 4 * (size_t)N, B.stream));
  B.a32 = Buf(sizeof(float) * (size_t)(n32 + N), B.stream);
  PDEB_CUDA(cudaMemsetAsync(B.a32.as<void>(), 0, sizeof(float) * (size_t)(n32 + N), B.stream));
  float* a32 = B.a32.as<float>();
  float* k32 = a32 + n32;
  const size_t khsz = B.bf16 ? sizeof(__nv_bfloat16) : sizeof(float);
  B.akh = Buf(khsz * (size_t)(N + nkh), B.stream);
  char* akh = B.akh.as<char>();
  for (int m = 0; m < count; ++m) {
    for (int l = 0; l < B.nlev[m]; ++l) {
      const int r = B.lev0[m] + l;
      BLevel& L = B.levels[r];
      L.x = a32 + x_off[r];
      L.b = a32 + b_off[r];
      L.r = a32 + r_off[r];
      if (L.kind != kDivk)
        L.kh = nullptr;
      else if (l == 0)
        L.kh = akh + khsz * (size_t)B.off[m];
      else
        L.kh = akh + khsz * (size_t)(N + kh_off[r]);
    }
  }
  // inputs into the packed FP64 arena (one copy per array and member)
  for (int m = 0; m < count; ++m) {
    const pdeb200_problem& hp = probs[m];
    const DevProblem& P = B.probs[m];
    const long long n0 = P.g.n;
    const cudaMemcpyKind kind = hp.mem_space == PDEB200_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    double* fm = B.f64 + B.off[m];
    if (hp.f) {
      PDEB_CUDA(cudaMemcpyAsync(fm, hp.f, sizeof(double) * n0, kind, B.stream));
    } else if (hp.f_const != 0.0) {
      const int blocks = (int)std::min<long long>((n0 + 255) / 256, 148LL * 8);
      k_fill<double><<<blocks, 256, 0, B.stream>>>(n0, fm, hp.f_const, nullptr);
    }
    if (P.coef_kind == kDivk) PDEB_CUDA(cudaMemcpyAsync(k64 + B.off[m], hp.k, sizeof(double) * n0, kind, B.stream));
    BMember& M = B.mem_tmpl[m];
    M.level0 = B.lev0[m];
    M.x64 = B.x64 + B.off[m];
    M.b64 = B.b64 + B.off[m];
    M.f64 = fm;
    M.k64 = P.coef_kind == kDivk ? k64 + B.off[m] : nullptr;
    M.k32 = P.coef_kind == kDivk ? k32 + B.off[m] : nullptr;
    M.p = a32 + p_off[m];
    M.q = a32 + q_off[m];
    M.e = a32 + e_off[m];
  }
  B.d_levels = Buf(sizeof(BLevel) * B.levels.size(), B.stream);
  PDEB_CUDA(cudaMemcpyAsync(B.d_levels.as<void>(), B.levels.data(), sizeof(BLevel) * B.levels.size(),
                            cudaMemcpyHostToDevice, B.stream));
  if (B.bf16)
    fill_hierarchy_k<__nv_bfloat16>(B, reinterpret_cast<__nv_bfloat16*>(akh), k32, k64);
  else
    fill_hierarchy_k<float>(B, reinterpret_cast<float*>(akh), k32, k64);
  B.d_mem = Buf(sizeof(BMember) * count, B.stream);
  B.d_active = Buf(sizeof(int), B.stream);
  PDEB_CUDA(cudaStreamSynchronize(B.stream));
}

// ---------------------------------------------------------------- autotune

std::string cache_key(const BatchPlan& B, const char* devname) {
  uint64_t h = 1469598103934665603ULL;
  auto mix = [&](long long v) {
    for (int q = 0; q < 8; ++q) {
      h ^= (uint64_t)((v >> (8 * q)) & 0xff);
      h *= 1099511628211ULL;
    }
  };
  for (int m = 0; m < B.count; ++m) {
    const GridDev& g = B.levels[B.lev0[m]].g;
    mix(g.nx);
    mix(g.ny);
    mix(g.nz);
    mix(B.levels[B.lev0[m]].kind);
  }
  mix(B.bf16 ? 1 : 0);
  std::ostringstream s;
  std::string dn(devname);
  for (auto& ch : dn)
    if (ch == ' ' || ch == '|') ch = '_';
  s << dn << "|" << B.count << "|" << std::hex << h;
  return s.str();
}

bool cache_lookup(const std::string& path, const std::string& key, BatchParams* p) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  bool found = false;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string k;
    BatchParams q = *p;
    if (!(ls >> k >> q.tile_x >> q.tile_y >> q.tile_z >> q.pre >> q.post >> q.inner_tol)) continue;
    if (k == key) {
      *p = q;
      found = true;  // the last entry for a key wins
    }
  }
  return found;
}

void cache_store(const std::string& path, const std::string& key, const BatchParams& p) {
  std::ofstream out(path, std::ios::app);
  if (!out) return;
  out << key << " " << p.tile_x << " " << p.tile_y << " " << p.tile_z << " " << p.pre << " " << p.post << " "
      << p.inner_tol << "\n";
}

double time_solve(BatchPlan& B) {
  build_schedule(B);
  solve_all(B, 1e-10);  // warm
  solve_all(B, 1e-10);
  return B.last_ms;
}

// Coordinate search over the schedule: tile shape of the 2D and 3D members,
// then the smoother sweeps, then the inner tolerance; each candidate is one
// timed solve of the whole batch.
void autotune(BatchPlan& B, const pdeb200_batch_options* o) {
  const char* env = std::getenv("PDEB200_TUNE_CACHE");
  const std::string path = o->tune_cache ? o->tune_cache : (env ? env : "");
  cudaDeviceProp prop;
  PDEB_CUDA(cudaGetDeviceProperties(&prop, B.dev));
  const std::string key = cache_key(B, prop.name);
  if (!path.empty() && cache_lookup(path, key, &B.prm)) {
    B.tuned_from_cache = true;
    return;
  }
  const auto t0 = std::chrono::steady_clock::now();
  bool has2 = false, has3 = false;
  for (int m = 0; m < B.count; ++m) (B.levels[B.lev0[m]].g.dim == 3 ? has3 : has2) = true;
  BatchParams best = B.prm;
  double best_ms = time_solve(B);
  auto trial = [&](const BatchParams& c) {
    B.prm = c;
    const double ms = time_solve(B);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  };
  if (has2) {
    const int shapes[][2] = {{32, 8}, {32, 16}, {32, 32}, {64, 16}, {64, 32}, {64, 64}};
    const BatchParams base = best;
    for (auto& sh : shapes) {
      if (sh[0] == base.tile_x && sh[1] == base.tile_y) continue;
      BatchParams c = base;
      c.tile_x = sh[0];
      c.tile_y = sh[1];
      trial(c);
    }
  }
  if (has3) {
    const BatchParams base = best;
    for (int tz : {4, 8, 16, 32}) {
      if (tz == base.tile_z) continue;
      BatchParams c = base;
      c.tile_z = tz;
      trial(c);
    }
  }
  {
    const BatchParams base = best;
    const int sm[][2] = {{1, 1}, {2, 2}, {2, 1}, {1, 2}, {3, 3}};
    for (auto& s : sm) {
      if (s[0] == base.pre && s[1] == base.post) continue;
      BatchParams c = base;
      c.pre = s[0];
      c.post = s[1];
      trial(c);
    }
  }
  {
    const BatchParams base = best;
    for (double it : {1e-3, 1e-4, 1e-5}) {
      if (it == base.inner_tol) continue;
      BatchParams c = base;
      c.inner_tol = it;
      trial(c);
    }
  }
  B.prm = best;
  B.tune_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (!path.empty()) cache_store(path, key, best);
}

void params_from_options(BatchParams* p, const pdeb200_batch_options* o) {
  if (o->tile_x > 0) p->tile_x = o->tile_x;
  if (o->tile_y > 0) p->tile_y = o->tile_y;
  if (o->tile_z > 0) p->tile_z = o->tile_z;
  if (o->pre_smooth > 0) p->pre = o->pre_smooth;
  if (o->post_smooth > 0) p->post = o->post_smooth;
  if (o->coarse_sweeps > 0) p->coarse_sweeps = o->coarse_sweeps;
  if (o->max_inner > 0) p->max_inner = o->max_inner;
  if (o->max_outer > 0) p->max_outer = o->max_outer;
  if (o->inner_tol > 0.0) p->inner_tol = o->inner_tol;
  if (p->tile_x != 32 && p->tile_x != 64) throw StatusFailure{PDEB200_ERR_INVALID, "tile_x must be 32 or 64"};
  if (p->tile_y < 1 || p->tile_y > 64) throw StatusFailure{PDEB200_ERR_INVALID, "tile_y must be in [1, 64]"};
  if (p->tile_z < 1 || p->tile_z > 1024) throw StatusFailure{PDEB200_ERR_INVALID, "tile_z must be in [1, 1024]"};
  if (p->pre > 8 || p->post > 8) throw StatusFailure{PDEB200_ERR_INVALID, "at most 8 smoothing sweeps"};
}

void copy_msg(char* dst, size_t len, const std::string& m) {
  if (!dst || len == 0) return;
  std::strncpy(dst, m.c_str(), len - 1);
  dst[len - 1] = '\0';
}

}  // namespace
}  // namespace pdeb

struct pdeb200_batch {
  pdeb::BatchPlan plan;
};

extern "C" {

void pdeb200_batch_default_options(pdeb200_batch_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
}

pdeb200_status pdeb200_batch_create(const pdeb200_problem* members, int32_t count, const pdeb200_batch_options* opt,
                                    pdeb200_batch** out, char* message, size_t message_len) {
  using namespace pdeb;
  if (out) *out = nullptr;
  copy_msg(message, message_len, "");
  if (!out) return PDEB200_ERR_INVALID;
  pdeb200_batch_options def;
  pdeb200_batch_default_options(&def);
  const pdeb200_batch_options* o = opt ? opt : &def;
  pdeb200_batch* b = nullptr;
  try {
    b = new pdeb200_batch();
    BatchPlan& B = b->plan;
    params_from_options(&B.prm, o);
    create_plan(B, members, count, o);
    if (o->autotune) autotune(B, o);
    build_schedule(B);
    *out = b;
    return PDEB200_OK;
  } catch (const StatusFailure& s) {
    copy_msg(message, message_len, s.what);
    delete b;
    return s.status;
  } catch (const CudaFailure& c) {
    copy_msg(message, message_len, c.what);
    cudaGetLastError();
    delete b;
    return PDEB200_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    copy_msg(message, message_len, "host memory exhausted");
    delete b;
    return PDEB200_ERR_OOM;
  }
}

int64_t pdeb200_batch_nodes(const pdeb200_batch* b) { return b ? b->plan.nodes : 0; }

int64_t pdeb200_batch_offset(const pdeb200_batch* b, int32_t member) {
  if (!b || member < 0 || member >= b->plan.count) return -1;
  return b->plan.off[member];
}

pdeb200_status pdeb200_batch_load_rhs(pdeb200_batch* b, const double* f, int32_t mem_space) {
  using namespace pdeb;
  if (!b || !f) return PDEB200_ERR_INVALID;
  BatchPlan& B = b->plan;
  const cudaMemcpyKind kind = mem_space == PDEB200_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (cudaSetDevice(B.dev) != cudaSuccess ||
      cudaMemcpyAsync(B.f64, f, sizeof(double) * (size_t)B.nodes, kind, B.stream) != cudaSuccess) {
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

pdeb200_status pdeb200_batch_solve(pdeb200_batch* b, double tol, pdeb200_report* reports,
                                   pdeb200_batch_stats* stats) {
  using namespace pdeb;
  if (!b || !(tol > 0.0)) return PDEB200_ERR_INVALID;
  BatchPlan& B = b->plan;
  const auto t0 = std::chrono::steady_clock::now();
  try {
    PDEB_CUDA(cudaSetDevice(B.dev));
    solve_all(B, tol);
  } catch (const StatusFailure& s) {
    if (reports) {
      for (int m = 0; m < B.count; ++m) {
        std::memset(&reports[m], 0, sizeof(pdeb200_report));
        set_report_msg(&reports[m], s.what);
      }
    }
    return s.status;
  } catch (const CudaFailure& c) {
    cudaGetLastError();
    if (reports) {
      for (int m = 0; m < B.count; ++m) {
        std::memset(&reports[m], 0, sizeof(pdeb200_report));
        set_report_msg(&reports[m], c.what);
      }
    }
    return PDEB200_ERR_CUDA;
  }
  const double total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  pdeb200_status first_bad = PDEB200_OK;
  int converged = 0;
  for (int m = 0; m < B.count; ++m) {
    const BMember& M = B.h_mem[m];
    if (M.status == PDEB200_OK)
      ++converged;
    else if (first_bad == PDEB200_OK)
      first_bad = (pdeb200_status)M.status;
    if (reports) {
      pdeb200_report& r = reports[m];
      std::memset(&r, 0, sizeof(r));
      r.iterations = M.inner_total;
      r.outer_iterations = M.outer > 0 ? M.outer - 1 : 0;
      r.converged = M.status == PDEB200_OK;
      r.kernel_launches = B.last_launches;
      r.residual_l2 = std::sqrt(M.rr_outer);
      r.rhs_l2 = std::sqrt(M.bb);
      r.rel_residual = M.bb > 0.0 ? std::sqrt(M.rr_outer / M.bb) : 0.0;
      r.device_ms = B.last_ms;
      r.total_ms = total_ms;
      set_report_msg(&r, pdeb200_status_string((pdeb200_status)M.status));
    }
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->members = B.count;
    stats->converged = converged;
    stats->cycles = B.last_cycles;
    stats->max_levels = B.lmax;
    stats->kernel_launches = B.last_launches;
    stats->tiles_level0 = B.full ? B.full->cnt[0] : 0;
    stats->nodes = B.nodes;
    size_t bytes = B.a64.bytes() + B.a32.bytes() + B.akh.bytes() + B.d_levels.bytes() + B.d_mem.bytes() +
                   (B.full ? B.full->tiles.bytes() + B.full->partials.bytes() : 0);
    for (const auto& P : B.probs)
      for (const auto& buf : P.owned) bytes += buf.bytes();
    for (const auto& buf : B.owned) bytes += buf.bytes();
    stats->device_bytes = (int64_t)bytes;
    stats->device_ms = B.last_ms;
    stats->tune_ms = B.tune_ms;
    stats->tuned_from_cache = B.tuned_from_cache ? 1 : 0;
    stats->graph = B.full && B.full->exec ? 1 : 0;
    stats->compactions = B.last_compactions;
  }
  return first_bad;
}

pdeb200_status pdeb200_batch_read(pdeb200_batch* b, double* out, int32_t mem_space) {
  using namespace pdeb;
  if (!b || !out) return PDEB200_ERR_INVALID;
  BatchPlan& B = b->plan;
  const cudaMemcpyKind kind = mem_space == PDEB200_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (cudaSetDevice(B.dev) != cudaSuccess ||
      cudaMemcpyAsync(out, B.x64, sizeof(double) * (size_t)B.nodes, kind, B.stream) != cudaSuccess ||
      cudaStreamSynchronize(B.stream) != cudaSuccess) {
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

pdeb200_status pdeb200_batch_read_member(pdeb200_batch* b, int32_t member, double* out, int32_t mem_space) {
  using namespace pdeb;
  if (!b || !out || member < 0 || member >= b->plan.count) return PDEB200_ERR_INVALID;
  BatchPlan& B = b->plan;
  const cudaMemcpyKind kind = mem_space == PDEB200_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t n = (size_t)B.probs[member].g.n;
  if (cudaSetDevice(B.dev) != cudaSuccess ||
      cudaMemcpyAsync(out, B.x64 + B.off[member], sizeof(double) * n, kind, B.stream) != cudaSuccess ||
      cudaStreamSynchronize(B.stream) != cudaSuccess) {
    cudaGetLastError();
    return PDEB200_ERR_CUDA;
  }
  return PDEB200_OK;
}

pdeb200_status pdeb200_batch_get_options(const pdeb200_batch* b, pdeb200_batch_options* o) {
  if (!b || !o) return PDEB200_ERR_INVALID;
  const pdeb::BatchPlan& B = b->plan;
  std::memset(o, 0, sizeof(*o));
  o->device = B.dev;
  o->tile_x = B.prm.tile_x;
  o->tile_y = B.prm.tile_y;
  o->tile_z = B.prm.tile_z;
  o->pre_smooth = B.prm.pre;
  o->post_smooth = B.prm.post;
  o->coarse_sweeps = B.prm.coarse_sweeps;
  o->max_inner = B.prm.max_inner;
  o->max_outer = B.prm.max_outer;
  o->bf16_coefficients = B.bf16 ? 1 : 0;
  o->no_graph = B.use_graph ? 0 : 1;
  o->no_compact = B.compact ? 0 : 1;
  o->inner_tol = B.prm.inner_tol;
  o->stream = B.own_stream ? nullptr : B.stream;
  return PDEB200_OK;
}

void pdeb200_batch_destroy(pdeb200_batch* b) {
  if (!b) return;
  cudaSetDevice(b->plan.dev);
  delete b;
}

}  // extern "C"
