// Drop-in implementation of the reference's CUDA backend entry points
// (pde_solver include/cuda_solver.h:8-9, src/backends/cuda/CudaSolve.h:7-10):
//
//   bool CudaIsAvailable(std::string* note);
//   SolveOutput SolvePDECuda(const SolveInput& input);
//   SolveOutput SolvePDETimeSeriesCuda(const SolveInput&, const FrameCallback&,
//                                      const ProgressCallback&);
//
// compiled inside pde_solver's build (it includes the reference's own
// pde_types.h and expression_eval.h) and linked against libpdeb200.so. It turns
// the parsed SolveInput into the POD problem of include/pdeb200.h: LaTeX right
// sides and coefficients are compiled once and evaluated at every node on the
// GPU (pdeb200_eval_expression, the language of ExpressionEvaluator), where the
// reference's CPU solver interprets them node by node
// (src/backends/cpu/solver.cpp:197, :834); boundary expressions go through
// the face form of the same evaluator, with the linear fallback of EvalExpr
// (cpu_utils.cpp:520-530). Then one C-ABI call solves on the GPU. Errors come back as SolveOutput.error strings, as the reference's
// backends report them.
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "cuda_solver.h"
#include "pde_types.h"
#include "pdeb200.h"
#include "progress.h"

using FrameCallback =
    std::function<bool(int frame, double time, const std::vector<double>& grid, const std::vector<double>* velocity)>;

namespace {

struct Materialised {
  pdeb200_problem prob{};
  std::vector<double> f, nodal, u0;
  std::vector<pdeb200_nonlinear_term> nonlinear;
  std::vector<double> face_arr[6][4];
  std::string error;
};

bool Unsupported(const SolveInput& in, std::string* why) {
  if (in.domain.coord_system != CoordinateSystem::Cartesian) {
    *why = "B200 backend supports Cartesian coordinates only";
    return true;
  }
  if (HasImplicitShape(in)) {
    *why = "B200 backend requires CPU fallback: implicit domain shape unsupported";
    return true;
  }
  if (!in.integrals.empty() || !in.nonlinear_derivatives.empty()) {
    *why = "B200 backend requires CPU fallback: integral or nonlinear derivative terms unsupported";
    return true;
  }
  if (in.nonlinear.size() > PDEB200_MAX_NONLINEAR) {
    *why = "B200 backend requires CPU fallback: more than 8 nonlinear terms";
    return true;
  }
  if (HasMixedDerivatives(in.pde) || HasHigherOrderDerivatives(in.pde)) {
    *why = "B200 backend requires CPU fallback: mixed or higher-order derivatives unsupported";
    return true;
  }
  if (!in.fields.empty()) {
    *why = "B200 backend requires CPU fallback: coupled fields unsupported";
    return true;
  }
  const std::vector<PiecewiseBoundaryCondition>* pw[6] = {&in.bc.left_piecewise,  &in.bc.right_piecewise,
                                                          &in.bc.bottom_piecewise, &in.bc.top_piecewise,
                                                          &in.bc.front_piecewise, &in.bc.back_piecewise};
  for (auto* p : pw)
    if (!p->empty()) {
      *why = "B200 backend requires CPU fallback: piecewise boundary conditions unsupported";
      return true;
    }
  return false;
}

// A LaTeX field at every node, compiled once and evaluated on the GPU by
// pdeb200_eval_expression (same language, guards and node coordinates as
// ExpressionEvaluator::Eval per node). Parse errors carry the reference's
// message after `prefix`.
bool EvalOnGrid(const std::string& latex, const pdeb200_problem& grid, int device, double* out, const char* prefix,
                std::string* error) {
  char msg[256];
  const pdeb200_status st = pdeb200_eval_expression(latex.c_str(), &grid, 0.0, device, out, PDEB200_MEM_HOST, msg,
                                                    sizeof(msg));
  if (st == PDEB200_OK) return true;
  *error = st == PDEB200_ERR_INVALID ? std::string(prefix) + msg
                                     : std::string("B200 expression evaluation failed: ") + pdeb200_status_string(st) +
                                           (msg[0] ? std::string(" (") + msg + ")" : std::string());
  return false;
}

bool Materialise(const SolveInput& in, Materialised* m, int device) {
  const Domain& d = in.domain;
  pdeb200_problem& p = m->prob;
  std::memset(&p, 0, sizeof(p));
  p.nx = d.nx;
  p.ny = d.ny;
  p.nz = d.nz > 1 ? d.nz : 1;
  p.xmin = d.xmin;
  p.xmax = d.xmax;
  p.ymin = d.ymin;
  p.ymax = d.ymax;
  p.zmin = d.zmin;
  p.zmax = d.zmax;
  p.mem_space = PDEB200_MEM_HOST;
  p.a = in.pde.a;
  p.b = in.pde.b;
  p.az = in.pde.az;
  p.c = in.pde.c;
  p.d = in.pde.d;
  p.dz = in.pde.dz;
  p.e = in.pde.e;
  p.f_const = in.pde.f;
  p.ut = in.pde.ut;
  if (d.nx < 3 || d.ny < 3 || (d.nz > 1 && d.nz < 3)) {
    m->error = "grid must be at least 3x3";
    return false;
  }
  if (!(d.xmax > d.xmin) || !(d.ymax > d.ymin) || (d.nz > 1 && !(d.zmax > d.zmin))) {
    m->error = "domain bounds are invalid";
    return false;
  }
  const int nz = p.nz;
  const long long n = (long long)p.nx * p.ny * nz;
  // right side (BuildRhs2D / the 3D sweep evaluate it per node)
  if (!in.pde.rhs_latex.empty()) {
    m->f.resize(n);
    if (!EvalOnGrid(in.pde.rhs_latex, p, device, m->f.data(), "invalid RHS expression: ", &m->error)) return false;
    p.f = m->f.data();
  }
  // variable coefficients (EvalCoefficient, src/coefficient_evaluator.cpp:99-105)
  if (HasVariableCoefficients(in.pde)) {
    const std::string* lat[7] = {&in.pde.a_latex, &in.pde.b_latex, &in.pde.az_latex, &in.pde.c_latex,
                                 &in.pde.d_latex, &in.pde.dz_latex, &in.pde.e_latex};
    const double cst[7] = {in.pde.a, in.pde.b, in.pde.az, in.pde.c, in.pde.d, in.pde.dz, in.pde.e};
    m->nodal.resize(7 * n);
    for (int q = 0; q < 7; ++q) {
      if (lat[q]->empty()) {
        std::fill(m->nodal.begin() + q * n, m->nodal.begin() + (q + 1) * n, cst[q]);
        continue;
      }
      if (!EvalOnGrid(*lat[q], p, device, m->nodal.data() + q * n, "invalid coefficient expression: ", &m->error))
        return false;
    }
    p.coef_kind = PDEB200_COEF_NODAL;
    p.nodal = m->nodal.data();
  }
  // faces
  const BoundaryCondition* bcs[6] = {&in.bc.left, &in.bc.right, &in.bc.bottom, &in.bc.top, &in.bc.front, &in.bc.back};
  for (int f = 0; f < 6; ++f) {
    const BoundaryCondition& bc = *bcs[f];
    pdeb200_face& F = p.face[f];
    F.kind = bc.kind == BCKind::Neumann ? PDEB200_BC_NEUMANN : bc.kind == BCKind::Robin ? PDEB200_BC_ROBIN
                                                                                        : PDEB200_BC_DIRICHLET;
    if (bc.kind != BCKind::Dirichlet && bc.kind != BCKind::Neumann && bc.kind != BCKind::Robin) {
      m->error = "B200 backend supports Dirichlet, Neumann and Robin boundaries";
      return false;
    }
    if (f >= 4 && nz <= 1) continue;
    const BoundaryCondition::Expression* ex[4] = {&bc.value, &bc.alpha, &bc.beta, &bc.gamma};
    const int w = f <= 1 ? p.ny : p.nx, h = f <= 3 ? nz : p.ny;
    for (int q = 0; q < 4; ++q) {
      std::vector<double>& arr = m->face_arr[f][q];
      arr.resize((size_t)w * h);
      const double lin[4] = {ex[q]->constant, ex[q]->x, ex[q]->y, ex[q]->z};
      char msg[256];
      const pdeb200_status st = pdeb200_eval_face_expression(ex[q]->latex.c_str(), lin, &p, f, 0.0, device,
                                                             arr.data(), PDEB200_MEM_HOST, msg, sizeof(msg));
      if (st != PDEB200_OK) {
        m->error = std::string("B200 boundary evaluation failed: ") + pdeb200_status_string(st) +
                   (msg[0] ? std::string(" (") + msg + ")" : std::string());
        return false;
      }
    }
    F.value_arr = m->face_arr[f][0].data();
    F.alpha_arr = m->face_arr[f][1].data();
    F.beta_arr = m->face_arr[f][2].data();
    F.gamma_arr = m->face_arr[f][3].data();
  }
  // pointwise nonlinear terms (NonlinearTerm, include/pde_types.h:96-100), same kind order
  for (const NonlinearTerm& t : in.nonlinear)
    m->nonlinear.push_back(pdeb200_nonlinear_term{static_cast<int32_t>(t.kind), t.power, t.coeff});
  p.n_nonlinear = (int32_t)m->nonlinear.size();
  p.nonlinear = m->nonlinear.empty() ? nullptr : m->nonlinear.data();
  if (!in.initial_grid.empty()) {
    if ((long long)in.initial_grid.size() != n) {
      m->error = "initial grid size mismatch";
      return false;
    }
    m->u0 = in.initial_grid;
    p.u0 = m->u0.data();
  }
  return true;
}

void FillOptions(const SolveInput& in, pdeb200_options* o) {
  pdeb200_default_options(o);
  o->method = static_cast<int32_t>(in.solver.method);  // SolveMethod order
  o->max_iter = in.solver.max_iter;
  o->tol = in.solver.tol;
  o->tol_mode = PDEB200_TOL_REFERENCE;
  o->sor_omega = in.solver.sor_omega;
  o->gmres_restart = in.solver.gmres_restart;
  o->mg_pre_smooth = in.solver.mg_pre_smooth;
  o->mg_post_smooth = in.solver.mg_post_smooth;
  o->mg_coarse_iters = in.solver.mg_coarse_iters;
  o->mg_max_levels = in.solver.mg_max_levels;
  o->gs_ordering = PDEB200_ORDER_LEXICOGRAPHIC;
  o->cancel = nullptr;  // SolveInput::cancel is ignored, as by the reference's CUDA backend
}

struct FrameTrampoline {
  const FrameCallback* cb;
  long long n;
  std::vector<double> scratch;
};

int32_t frame_thunk(int32_t frame, double time, const double* grid, void* user) {
  FrameTrampoline* t = static_cast<FrameTrampoline*>(user);
  t->scratch.assign(grid, grid + t->n);
  return (*t->cb)(frame, time, t->scratch, nullptr) ? 1 : 0;
}

}  // namespace

bool CudaIsAvailable(std::string* note) {
  char buf[256] = {0};
  const int ok = pdeb200_probe(buf, sizeof(buf));
  if (note) *note = buf;
  return ok != 0;
}

SolveOutput SolvePDECuda(const SolveInput& input) {
  std::string why;
  if (std::abs(input.pde.ut) > 1e-12 || std::abs(input.pde.utt) > 1e-12)
    return {"time-dependent PDEs require the time-series solver", {}};
  if (Unsupported(input, &why)) return {why, {}};
  std::string note;
  if (!CudaIsAvailable(&note)) return {"CUDA unavailable: " + note, {}};
  Materialised m;
  if (!Materialise(input, &m, 0)) return {m.error, {}};
  pdeb200_options o;
  FillOptions(input, &o);
  const bool krylov = input.solver.method == SolveMethod::CG || input.solver.method == SolveMethod::BiCGStab ||
                      input.solver.method == SolveMethod::GMRES;
  // the reference's order: linearity before the CG symmetry check (src/backends/cpu/solver.cpp:502,550)
  if (!input.nonlinear.empty() && krylov) return {"Krylov solvers require linear PDEs", {}};
  if (!input.nonlinear.empty() && input.solver.method == SolveMethod::MultigridVcycle)
    return {"Multigrid requires linear PDEs", {}};
  if (input.solver.method == SolveMethod::CG && (HasVariableCoefficients(input.pde) ||
                                                 std::abs(input.pde.c) > 1e-12 || std::abs(input.pde.d) > 1e-12))
    return {"CG requires symmetric operators with constant coefficients (no convection/mixed/higher-order terms)", {}};
  SolveOutput out;
  out.grid.resize((size_t)m.prob.nx * m.prob.ny * m.prob.nz);
  pdeb200_report rep;
  const pdeb200_status st = pdeb200_solve(&m.prob, &o, out.grid.data(), &rep);
  if (st == PDEB200_OK) return out;
  if (st == PDEB200_ERR_NOT_CONVERGED && !krylov && input.solver.method != SolveMethod::MultigridVcycle)
    return out;  // relaxation returns its last iterate without an error (relaxation.cpp:296-307)
  std::string msg = rep.message[0] ? rep.message : pdeb200_status_string(st);
  if (krylov && (st == PDEB200_ERR_NOT_CONVERGED || st == PDEB200_ERR_BREAKDOWN))
    msg = "CUDA Krylov solver failed to converge";
  return {msg, {}};
}

SolveOutput SolvePDETimeSeriesCuda(const SolveInput& input, const FrameCallback& on_frame,
                                   const ProgressCallback& progress) {
  std::string why;
  if (Unsupported(input, &why)) return {why, {}};
  if (std::abs(input.pde.utt) > 1e-12) return {"B200 time series supports first-order (u_t) problems", {}};
  if (std::abs(input.pde.ut) <= 1e-12) return {"time-dependent solve requires u_t or u_tt term", {}};
  if (input.time.integrator != TimeIntegrator::ForwardEuler)
    return {"B200 time series supports forward Euler", {}};
  Materialised m;
  if (!Materialise(input, &m, 0)) return {m.error, {}};
  pdeb200_time_options t{};
  t.t_start = input.time.t_start;
  t.dt = input.time.dt;
  t.frames = input.time.frames;
  t.frame_stride = 1;
  t.device = 0;
  FrameTrampoline tr{&on_frame, (long long)m.prob.nx * m.prob.ny * m.prob.nz, {}};
  SolveOutput out;
  out.grid.resize((size_t)tr.n);
  pdeb200_report rep;
  if (progress) progress("solve", 0.0);
  const pdeb200_status st =
      pdeb200_time_series(&m.prob, &t, on_frame ? frame_thunk : nullptr, &tr, out.grid.data(), &rep);
  if (progress) progress("solve", 1.0);
  if (st != PDEB200_OK) return {rep.message[0] ? rep.message : pdeb200_status_string(st), {}};
  return out;
}
