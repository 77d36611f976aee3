// Test infrastructure only (oracle). A C ABI around the reference's own CPU
// solver, compiled from the reference sources by oracle/Makefile into
// oracle/_ref/libpderef.so. tests/ and bench.py's CPU baseline call it through
// ctypes to produce the fields the B200 library must reproduce.
//
// It builds a SolveInput exactly the way src/self_test.cpp:110-125 does
// (constant or LaTeX expressions, Cartesian domain) and calls the reference
// entry points unchanged:
//   SolveWithBackend(..., BackendKind::CPU, ...)   src/backend_solve.cpp:53
//   SolvePDETimeSeries                             src/backends/cpu/solver.cpp:989
//   ProjectVelocity2D / ProjectVelocity3D          src/pressure_projection.cpp:255,698
//   ComputeResidualNorms                           src/residual.cpp:153
//   RunSelfTest                                    src/self_test.cpp:224
//   WriteVtkStructuredPoints / WriteVtkXmlImageData src/vtk_writer.cpp:28,176
// Built with PDEREF_DROPIN (oracle/_ref/libdropin.so) it also drives the
// reference's SolveWithBackend with the CUDA backend compiled in and served by
// the B200 shim (pde_solver_b200/shim/cuda_solver_shim.cpp).
#include <omp.h>

#include <cstring>
#include <string>
#include <vector>

#include "backend.h"
#include "expression_eval.h"
#include "pde_types.h"
#include "pdeb200.h"
#include "pressure_projection.h"
#include "residual.h"
#include "self_test.h"
#include "solver.h"
#include "vtk_io.h"
#ifdef PDEREF_DROPIN
#include "cuda_solver.h"
SolveOutput SolvePDETimeSeriesCuda(const SolveInput& input, const FrameCallback& on_frame,
                                   const ProgressCallback& progress);
#endif

namespace {

void CopyError(const std::string& s, char* err, size_t len) {
  if (!err || len == 0) return;
  std::strncpy(err, s.c_str(), len - 1);
  err[len - 1] = '\0';
}

BoundaryCondition FaceToBC(const pdeb200_face& f) {
  BoundaryCondition bc;
  bc.kind = f.kind == PDEB200_BC_NEUMANN ? BCKind::Neumann
            : f.kind == PDEB200_BC_ROBIN ? BCKind::Robin
                                          : BCKind::Dirichlet;
  bc.value.constant = f.value;
  bc.alpha.constant = f.alpha;
  bc.beta.constant = f.beta;
  bc.gamma.constant = f.gamma;
  return bc;
}

// coef_latex: optional array of 7 strings (a,b,az,c,d,dz,e); NULL entries keep constants.
bool BuildInput(const pdeb200_problem* p, const char* rhs_latex, const char* const* coef_latex,
                SolveInput* in, std::string* error) {
  if (p->coef_kind != PDEB200_COEF_CONST) {
    *error = "reference supports constant or LaTeX coefficients only";
    return false;
  }
  for (int f = 0; f < 6; ++f) {
    if (p->face[f].value_arr || p->face[f].alpha_arr || p->face[f].beta_arr || p->face[f].gamma_arr) {
      *error = "reference driver takes constant boundary values only";
      return false;
    }
  }
  if (p->f) {
    *error = "reference takes the RHS as LaTeX or a constant";
    return false;
  }
  in->domain.xmin = p->xmin;
  in->domain.xmax = p->xmax;
  in->domain.ymin = p->ymin;
  in->domain.ymax = p->ymax;
  in->domain.zmin = p->zmin;
  in->domain.zmax = p->zmax;
  in->domain.nx = p->nx;
  in->domain.ny = p->ny;
  in->domain.nz = p->nz <= 1 ? 1 : p->nz;
  in->pde.a = p->a;
  in->pde.b = p->b;
  in->pde.az = p->az;
  in->pde.c = p->c;
  in->pde.d = p->d;
  in->pde.dz = p->dz;
  in->pde.e = p->e;
  in->pde.f = p->f_const;
  in->pde.ut = p->ut;
  if (rhs_latex) in->pde.rhs_latex = rhs_latex;
  if (coef_latex) {
    std::string* slots[7] = {&in->pde.a_latex, &in->pde.b_latex, &in->pde.az_latex,
                             &in->pde.c_latex, &in->pde.d_latex, &in->pde.dz_latex,
                             &in->pde.e_latex};
    for (int i = 0; i < 7; ++i) {
      if (coef_latex[i]) *slots[i] = coef_latex[i];
    }
  }
  in->bc.left = FaceToBC(p->face[0]);
  in->bc.right = FaceToBC(p->face[1]);
  in->bc.bottom = FaceToBC(p->face[2]);
  in->bc.top = FaceToBC(p->face[3]);
  in->bc.front = FaceToBC(p->face[4]);
  in->bc.back = FaceToBC(p->face[5]);
  if (p->u0) {
    const size_t n = static_cast<size_t>(p->nx) * p->ny * (p->nz <= 1 ? 1 : p->nz);
    in->initial_grid.assign(p->u0, p->u0 + n);
  }
  for (int t = 0; t < p->n_nonlinear; ++t) {
    NonlinearTerm nt;
    nt.kind = static_cast<NonlinearKind>(p->nonlinear[t].kind);
    nt.coeff = p->nonlinear[t].coeff;
    nt.power = p->nonlinear[t].power;
    in->nonlinear.push_back(nt);
  }
  return true;
}

void ApplyOptions(const pdeb200_options* o, SolveInput* in) {
  switch (o->method) {
    case PDEB200_JACOBI: in->solver.method = SolveMethod::Jacobi; break;
    case PDEB200_GAUSS_SEIDEL: in->solver.method = SolveMethod::GaussSeidel; break;
    case PDEB200_SOR: in->solver.method = SolveMethod::SOR; break;
    case PDEB200_CG: in->solver.method = SolveMethod::CG; break;
    case PDEB200_BICGSTAB: in->solver.method = SolveMethod::BiCGStab; break;
    case PDEB200_GMRES: in->solver.method = SolveMethod::GMRES; break;
    default: in->solver.method = SolveMethod::MultigridVcycle; break;
  }
  in->solver.max_iter = o->max_iter;
  in->solver.tol = o->tol;
  in->solver.sor_omega = o->sor_omega;
  in->solver.gmres_restart = o->gmres_restart;
  in->solver.mg_pre_smooth = o->mg_pre_smooth;
  in->solver.mg_post_smooth = o->mg_post_smooth;
  in->solver.mg_coarse_iters = o->mg_coarse_iters;
  in->solver.mg_max_levels = o->mg_max_levels;
  in->solver.residual_interval = 0;
}

}  // namespace

extern "C" {

void pderef_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int pderef_max_threads(void) { return omp_get_max_threads(); }

// Steady solve through the reference's backend dispatch on the CPU backend.
// Returns 0 on success; out receives nx*ny*nz values; resid gets the reference's
// own post-solve residual norms (MaybeComputeResiduals, src/backend_solve.cpp:40-50).
int pderef_solve(const pdeb200_problem* p, const char* rhs_latex, const char* const* coef_latex,
                 const pdeb200_options* o, double* out, double* resid_l2, double* resid_linf,
                 char* err, size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, coef_latex, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  ApplyOptions(o, &in);
  BackendKind selected = BackendKind::CPU;
  std::string note;
  SolveOutput res = SolveWithBackend(in, BackendKind::CPU, &selected, &note);
  if (!res.error.empty()) {
    CopyError(res.error, err, err_len);
    return 2;
  }
  std::memcpy(out, res.grid.data(), res.grid.size() * sizeof(double));
  if (resid_l2) *resid_l2 = res.residual_l2;
  if (resid_linf) *resid_linf = res.residual_linf;
  return 0;
}

// Forward-Euler time series (SolvePDETimeSeries). frames_out (optional) receives
// every frame back to back; out receives the last frame.
int pderef_time_series(const pdeb200_problem* p, const char* rhs_latex, double t_start, double dt,
                       int frames, double* out, double* frames_out, char* err, size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, nullptr, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  in.time.enabled = true;
  in.time.t_start = t_start;
  in.time.dt = dt;
  in.time.frames = frames;
  const size_t n = static_cast<size_t>(p->nx) * p->ny * (p->nz <= 1 ? 1 : p->nz);
  FrameCallback cb = [&](int frame, double, const std::vector<double>& grid,
                         const std::vector<double>*) -> bool {
    if (frames_out) std::memcpy(frames_out + static_cast<size_t>(frame) * n, grid.data(), n * sizeof(double));
    return true;
  };
  SolveOutput res = SolvePDETimeSeries(in, cb, ProgressCallback());
  if (!res.error.empty()) {
    CopyError(res.error, err, err_len);
    return 2;
  }
  std::memcpy(out, res.grid.data(), n * sizeof(double));
  return 0;
}

// Reference residual norms of a given grid (ComputeResidualNorms).
int pderef_residual_norms(const pdeb200_problem* p, const char* rhs_latex, const double* grid,
                          double* l2, double* linf, char* err, size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, nullptr, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  const size_t n = static_cast<size_t>(p->nx) * p->ny * (p->nz <= 1 ? 1 : p->nz);
  std::vector<double> g(grid, grid + n);
  ResidualNorms norms;
  if (!ComputeResidualNorms(in, g, &norms, &error)) {
    CopyError(error, err, err_len);
    return 2;
  }
  *l2 = norms.l2;
  *linf = norms.linf;
  return 0;
}

// Evaluates a LaTeX expression at every node (x fastest), as BuildRhs2D and the
// 3D sweep do per node (solver.cpp:197, :834).
int pderef_materialize(const char* latex, int nx, int ny, int nz, double xmin, double xmax,
                       double ymin, double ymax, double zmin, double zmax, double t, double* out,
                       char* err, size_t err_len) {
  ExpressionEvaluator ev = ExpressionEvaluator::ParseLatex(latex);
  if (!ev.ok()) {
    CopyError(ev.error(), err, err_len);
    return 1;
  }
  const int nzz = nz <= 1 ? 1 : nz;
  const double dx = (xmax - xmin) / (nx - 1);
  const double dy = (ymax - ymin) / (ny - 1);
  const double dz = nzz > 1 ? (zmax - zmin) / (nzz - 1) : 0.0;
  for (int k = 0; k < nzz; ++k) {
    for (int j = 0; j < ny; ++j) {
      for (int i = 0; i < nx; ++i) {
        const double z = nzz > 1 ? zmin + k * dz : 0.0;
        out[(static_cast<size_t>(k) * ny + j) * nx + i] = ev.Eval(xmin + i * dx, ymin + j * dy, z, t);
      }
    }
  }
  return 0;
}

// ProjectVelocity2D / 3D (collocated grid). nz <= 1 selects 2D.
int pderef_project(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double* u,
                   double* v, double* w, double* pressure, int max_iter, double tol,
                   int fix_corner, double* report /* [iters, residual, maxdiv0, maxdiv1, l2div0, l2div1] */) {
  ProjectionConfig cfg;
  cfg.max_iter = max_iter;
  cfg.tol = tol;
  cfg.fix_pressure_corner = fix_corner != 0;
  ProjectionResult r;
  if (nz <= 1) {
    const size_t n = static_cast<size_t>(nx) * ny;
    VelocityField2D vel;
    vel.nx = nx;
    vel.ny = ny;
    vel.dx = dx;
    vel.dy = dy;
    vel.u.assign(u, u + n);
    vel.v.assign(v, v + n);
    std::vector<double> p(pressure, pressure + n);
    r = ProjectVelocity2D(vel, dt, &p, cfg);
    std::memcpy(u, vel.u.data(), n * sizeof(double));
    std::memcpy(v, vel.v.data(), n * sizeof(double));
    std::memcpy(pressure, p.data(), n * sizeof(double));
  } else {
    const size_t n = static_cast<size_t>(nx) * ny * nz;
    VelocityField3D vel;
    vel.nx = nx;
    vel.ny = ny;
    vel.nz = nz;
    vel.dx = dx;
    vel.dy = dy;
    vel.dz = dz;
    vel.u.assign(u, u + n);
    vel.v.assign(v, v + n);
    vel.w.assign(w, w + n);
    std::vector<double> p(pressure, pressure + n);
    r = ProjectVelocity3D(vel, dt, &p, cfg);
    std::memcpy(u, vel.u.data(), n * sizeof(double));
    std::memcpy(v, vel.v.data(), n * sizeof(double));
    std::memcpy(w, vel.w.data(), n * sizeof(double));
    std::memcpy(pressure, p.data(), n * sizeof(double));
  }
  if (report) {
    report[0] = r.poisson_iterations;
    report[1] = r.poisson_residual;
    report[2] = r.max_divergence_before;
    report[3] = r.max_divergence_after;
    report[4] = r.l2_divergence_before;
    report[5] = r.l2_divergence_after;
  }
  return r.success ? 0 : 2;
}

// The reference's own analytic self-test (src/self_test.cpp:224-411); returns
// 1 when any case fails.
int pderef_self_test(void) { return RunSelfTest(); }

// The reference's VTK writers on a Domain built from the problem's geometry
// (nz <= 1 gives Domain::nz = 1). derived != 0 passes the derived fields the
// way the reference CLI does (BuildDerivedFieldVectors, src/main.cpp:255-288).
Domain DomainOf(const pdeb200_problem* p) {
  Domain d;
  d.nx = p->nx;
  d.ny = p->ny;
  d.nz = p->nz <= 1 ? 1 : p->nz;
  d.xmin = p->xmin;
  d.xmax = p->xmax;
  d.ymin = p->ymin;
  d.ymax = p->ymax;
  d.zmin = p->zmin;
  d.zmax = p->zmax;
  return d;
}

int pderef_write_vtk(const char* path, const pdeb200_problem* p, const double* grid, char* err, size_t err_len) {
  const Domain d = DomainOf(p);
  const std::vector<double> g(grid, grid + static_cast<size_t>(d.nx) * d.ny * d.nz);
  VtkWriteResult r = WriteVtkStructuredPoints(path, d, g);
  if (!r.ok) {
    CopyError(r.error, err, err_len);
    return 1;
  }
  return 0;
}

int pderef_write_vti(const char* path, const pdeb200_problem* p, const double* grid, int derived, char* err,
                     size_t err_len) {
  const Domain d = DomainOf(p);
  const std::vector<double> g(grid, grid + static_cast<size_t>(d.nx) * d.ny * d.nz);
  std::vector<std::vector<double>> data;
  std::vector<std::string> names;
  if (derived) {
    DerivedFields f = ComputeDerivedFields(d, g, p->a, p->b, p->az);
    data.push_back(f.gradient_x);
    names.push_back("gradient_x");
    data.push_back(f.gradient_y);
    names.push_back("gradient_y");
    if (d.nz > 1) {
      data.push_back(f.gradient_z);
      names.push_back("gradient_z");
    }
    data.push_back(f.laplacian);
    names.push_back("laplacian");
    data.push_back(f.flux_x);
    names.push_back("flux_x");
    data.push_back(f.flux_y);
    names.push_back("flux_y");
    if (d.nz > 1) {
      data.push_back(f.flux_z);
      names.push_back("flux_z");
    }
    data.push_back(f.energy_norm);
    names.push_back("energy_norm");
  }
  VtkWriteResult r = WriteVtkXmlImageData(path, d, g, derived ? &data : nullptr, derived ? &names : nullptr);
  if (!r.ok) {
    CopyError(r.error, err, err_len);
    return 1;
  }
  return 0;
}

#ifdef PDEREF_DROPIN
// Drop-in harness: the same SolveInput through the reference's dispatch with
// the CUDA backend compiled in (USE_CUDA) and served by the B200 shim.
int dropin_solve_with_backend(const pdeb200_problem* p, const char* rhs_latex, const char* const* coef_latex,
                              const char* const* face_value_latex, const pdeb200_options* o, int backend,
                              double* out, double* resid_l2, double* resid_linf, int* selected, char* err,
                              size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, coef_latex, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  if (face_value_latex) {
    BoundaryCondition* bcs[6] = {&in.bc.left, &in.bc.right, &in.bc.bottom, &in.bc.top, &in.bc.front, &in.bc.back};
    for (int f = 0; f < 6; ++f)
      if (face_value_latex[f]) bcs[f]->value.latex = face_value_latex[f];
  }
  ApplyOptions(o, &in);
  BackendKind sel = BackendKind::CPU;
  std::string note;
  SolveOutput res = SolveWithBackend(in, backend == 1 ? BackendKind::CUDA : BackendKind::CPU, &sel, &note);
  if (selected) *selected = sel == BackendKind::CUDA ? 1 : 0;
  if (!res.error.empty()) {
    CopyError(res.error, err, err_len);
    return 2;
  }
  std::memcpy(out, res.grid.data(), res.grid.size() * sizeof(double));
  if (resid_l2) *resid_l2 = res.residual_l2;
  if (resid_linf) *resid_linf = res.residual_linf;
  return 0;
}

// SolvePDECuda directly (the reference's capability gate keeps CUDA to 2D).
int dropin_solve_cuda(const pdeb200_problem* p, const char* rhs_latex, const char* const* coef_latex,
                      const char* const* face_value_latex, const pdeb200_options* o, double* out, char* err,
                      size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, coef_latex, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  if (face_value_latex) {
    BoundaryCondition* bcs[6] = {&in.bc.left, &in.bc.right, &in.bc.bottom, &in.bc.top, &in.bc.front, &in.bc.back};
    for (int f = 0; f < 6; ++f)
      if (face_value_latex[f]) bcs[f]->value.latex = face_value_latex[f];
  }
  ApplyOptions(o, &in);
  SolveOutput res = SolvePDECuda(in);
  if (!res.error.empty()) {
    CopyError(res.error, err, err_len);
    return 2;
  }
  std::memcpy(out, res.grid.data(), res.grid.size() * sizeof(double));
  return 0;
}

int dropin_time_series_cuda(const pdeb200_problem* p, const char* rhs_latex, double t_start, double dt, int frames,
                            double* out, double* frames_out, char* err, size_t err_len) {
  SolveInput in;
  std::string error;
  if (!BuildInput(p, rhs_latex, nullptr, &in, &error)) {
    CopyError(error, err, err_len);
    return 1;
  }
  in.time.enabled = true;
  in.time.t_start = t_start;
  in.time.dt = dt;
  in.time.frames = frames;
  const size_t n = static_cast<size_t>(p->nx) * p->ny * (p->nz <= 1 ? 1 : p->nz);
  FrameCallback cb = [&](int frame, double, const std::vector<double>& grid, const std::vector<double>*) -> bool {
    if (frames_out) std::memcpy(frames_out + static_cast<size_t>(frame) * n, grid.data(), n * sizeof(double));
    return true;
  };
  SolveOutput res = SolvePDETimeSeriesCuda(in, cb, ProgressCallback());
  if (!res.error.empty()) {
    CopyError(res.error, err, err_len);
    return 2;
  }
  std::memcpy(out, res.grid.data(), n * sizeof(double));
  return 0;
}

int dropin_probe(char* note, size_t len) {
  std::string s;
  const bool ok = CudaIsAvailable(&s);
  CopyError(s, note, len);
  return ok ? 1 : 0;
}
#endif

}  // extern "C"
