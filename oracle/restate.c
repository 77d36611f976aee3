/* Test infrastructure only (the oracle): plain-C restatement of the
 * reference's structured-grid solve path. tests/, smoke() and the CPU
 * baseline of bench.py compare libpdeb200.so against it; nothing in the
 * product links or calls it.
 *
 * Expression order follows the reference line by line where the reference
 * has the computation, so that the restatement reproduces oracle/_ref
 * (the reference compiled from its own sources) bit for bit on the cases the
 * reference covers; tests/test_oracle_pins.py checks that.
 *
 * Reference files cited (paths inside nathanielasun/pde_solver):
 *   src/backends/cpu/solver.cpp, src/backends/cpu/cpu_utils.cpp,
 *   src/backends/cpu/solvers/{relaxation,krylov,multigrid}.cpp,
 *   src/residual.cpp, src/pressure_projection.cpp.
 */
#include "restate.h"

#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ grid */

enum { LEFT = 0, RIGHT, BOTTOM, TOP, FRONT, BACK };

typedef struct {
  const pdeb200_problem* p;
  int nx, ny, nz, dim;
  long n;
  double xmin, ymin, zmin, dx, dy, dz;
  /* face parameters materialised per face node (face-local index) */
  int fsize[6];
  double* val[6];
  double* al[6];
  double* be[6];
  double* ga[6];
} Grid;

static inline long ID(const Grid* g, int i, int j, int k) {
  return ((long)k * g->ny + j) * g->nx + i;
}

static void set_msg(pdeb200_report* r, const char* m) {
  if (r) {
    strncpy(r->message, m, sizeof(r->message) - 1);
    r->message[sizeof(r->message) - 1] = 0;
  }
}

static double* mat_face(const double* arr, double c, int n) {
  double* out = (double*)malloc(sizeof(double) * (size_t)n);
  for (int i = 0; i < n; ++i) out[i] = arr ? arr[i] : c;
  return out;
}

/* include/safe_math.h:134-170 spacing, src/backends/cpu/solver.cpp:462-467 */
static int grid_init(Grid* g, const pdeb200_problem* p) {
  memset(g, 0, sizeof(*g));
  g->p = p;
  g->nx = p->nx;
  g->ny = p->ny;
  g->nz = p->nz <= 1 ? 1 : p->nz;
  g->dim = p->nz > 1 ? 3 : 2;
  if (g->nx < 3 || g->ny < 3 || (g->dim == 3 && g->nz < 3)) return PDEB200_ERR_INVALID;
  if (!(p->xmax > p->xmin) || !(p->ymax > p->ymin) || (g->dim == 3 && !(p->zmax > p->zmin)))
    return PDEB200_ERR_INVALID;
  g->n = (long)g->nx * g->ny * g->nz;
  g->xmin = p->xmin;
  g->ymin = p->ymin;
  g->zmin = p->zmin;
  g->dx = (p->xmax - p->xmin) / (double)(g->nx - 1);
  g->dy = (p->ymax - p->ymin) / (double)(g->ny - 1);
  g->dz = g->dim == 3 ? (p->zmax - p->zmin) / (double)(g->nz - 1) : 0.0;
  const int fs[6] = {g->ny * g->nz, g->ny * g->nz, g->nx * g->nz, g->nx * g->nz,
                     g->nx * g->ny, g->nx * g->ny};
  for (int f = 0; f < 6; ++f) {
    g->fsize[f] = fs[f];
    const pdeb200_face* fc = &p->face[f];
    g->val[f] = mat_face(fc->value_arr, fc->value, fs[f]);
    g->al[f] = mat_face(fc->alpha_arr, fc->alpha, fs[f]);
    g->be[f] = mat_face(fc->beta_arr, fc->beta, fs[f]);
    g->ga[f] = mat_face(fc->gamma_arr, fc->gamma, fs[f]);
  }
  return PDEB200_OK;
}

static void grid_free(Grid* g) {
  for (int f = 0; f < 6; ++f) {
    free(g->val[f]);
    free(g->al[f]);
    free(g->be[f]);
    free(g->ga[f]);
  }
}

static int face_active(const Grid* g, int f) { return g->dim == 3 || f < FRONT; }
static int face_kind(const Grid* g, int f) { return g->p->face[f].kind; }

/* --------------------------------------------------------- coefficients */

typedef struct {
  double c, xm, xp, ym, yp, zm, zp;
} Stencil;

/* Stencil weights of interior node (i,j,k).
 * CONST / NODAL: src/backends/cpu/solver.cpp:855-866 (3D), cpu_utils.cpp:421-433 (2D).
 * DIVK: divergence form with face-averaged k; constant k reproduces a=b=az=-k. */
static void node_stencil(const Grid* g, int i, int j, int k, Stencil* s) {
  const pdeb200_problem* p = g->p;
  const double dx = g->dx, dy = g->dy, dz = g->dz;
  const long id = ID(g, i, j, k);
  if (p->coef_kind == PDEB200_COEF_DIVK) {
    const double* K = p->k;
    const double kc = K[id];
    const double kxm = 0.5 * (kc + K[id - 1]), kxp = 0.5 * (kc + K[id + 1]);
    const double kym = 0.5 * (kc + K[id - g->nx]), kyp = 0.5 * (kc + K[id + g->nx]);
    const double cx = p->c / (2.0 * dx), dyc = p->d / (2.0 * dy);
    s->xm = -kxm / (dx * dx) - cx;
    s->xp = -kxp / (dx * dx) + cx;
    s->ym = -kym / (dy * dy) - dyc;
    s->yp = -kyp / (dy * dy) + dyc;
    double center = (kxm + kxp) / (dx * dx) + (kym + kyp) / (dy * dy);
    if (g->dim == 3) {
      const long sz = (long)g->nx * g->ny;
      const double kzm = 0.5 * (kc + K[id - sz]), kzp = 0.5 * (kc + K[id + sz]);
      const double dzc = p->dz / (2.0 * dz);
      s->zm = -kzm / (dz * dz) - dzc;
      s->zp = -kzp / (dz * dz) + dzc;
      center = center + (kzm + kzp) / (dz * dz);
    } else {
      s->zm = s->zp = 0.0;
    }
    s->c = center + p->e;
    return;
  }
  double a = p->a, b = p->b, az = p->az, c = p->c, d = p->d, dzv = p->dz, e = p->e;
  if (p->coef_kind == PDEB200_COEF_NODAL) {
    const double* A = p->nodal;
    a = A[id];
    b = A[g->n + id];
    az = A[2 * g->n + id];
    c = A[3 * g->n + id];
    d = A[4 * g->n + id];
    dzv = A[5 * g->n + id];
    e = A[6 * g->n + id];
  }
  const double ax = a / (dx * dx);
  const double by = b / (dy * dy);
  const double cx = c / (2.0 * dx);
  const double dyc = d / (2.0 * dy);
  s->xp = ax + cx;
  s->xm = ax - cx;
  s->yp = by + dyc;
  s->ym = by - dyc;
  if (g->dim == 3) {
    const double cz = az / (dz * dz);
    const double dzc = dzv / (2.0 * dz);
    s->zp = cz + dzc;
    s->zm = cz - dzc;
    s->c = -2.0 * ax - 2.0 * by - 2.0 * cz + e;
  } else {
    s->zp = s->zm = 0.0;
    s->c = -2.0 * ax - 2.0 * by + e;
  }
}

static inline double f_at(const Grid* g, long id) {
  return g->p->f ? g->p->f[id] : g->p->f_const;
}

/* EvalNonlinear (relaxation.cpp:27-45, solver.cpp:234-256): sum of
 * coeff * g(u) in term order, g = u^power, sin, cos, exp, |u|. */
static double eval_nonlinear(const pdeb200_problem* p, double u) {
  double value = 0.0;
  for (int t = 0; t < p->n_nonlinear; ++t) {
    const pdeb200_nonlinear_term* nt = &p->nonlinear[t];
    switch (nt->kind) {
      case PDEB200_NL_POWER: value += nt->coeff * pow(u, (double)nt->power); break;
      case PDEB200_NL_SIN: value += nt->coeff * sin(u); break;
      case PDEB200_NL_COS: value += nt->coeff * cos(u); break;
      case PDEB200_NL_EXP: value += nt->coeff * exp(u); break;
      default: value += nt->coeff * fabs(u); break;
    }
  }
  return value;
}

/* (f + integral) + nonlinear, the reference's sum with no integral term
 * (relaxation.cpp:281, solver.cpp:948, residual.cpp:487). */
static inline double f_nl(const Grid* g, long id, double u) {
  const double f = f_at(g, id);
  return g->p->n_nonlinear ? f + eval_nonlinear(g->p, u) : f;
}

/* Neighbour sum in the reference's order (solver.cpp:892-898, cpu_utils.cpp:428-433). */
static inline double nb_sum(const Grid* g, const Stencil* s, const double* u, long id) {
  double v = s->xp * u[id + 1] + s->xm * u[id - 1] + s->yp * u[id + g->nx] + s->ym * u[id - g->nx];
  if (g->dim == 3) {
    const long sz = (long)g->nx * g->ny;
    v = v + s->zp * u[id + sz] + s->zm * u[id - sz];
  }
  return v;
}

static int check_center(const Grid* g) {
  /* constant-coefficient degenerate check (solver.cpp:733-737, relaxation.cpp:120-123) */
  if (g->p->coef_kind == PDEB200_COEF_CONST) {
    Stencil s;
    if (g->nx >= 3 && g->ny >= 3) {
      node_stencil(g, 1, 1, g->dim == 3 ? 1 : 0, &s);
      if (fabs(s.c) < 1e-12) return PDEB200_ERR_DEGENERATE;
    }
  }
  return PDEB200_OK;
}

/* ----------------------------------------------------- boundary closures */

/* Face node (face-local index) for node (i,j,k) on face f. */
static inline int flocal(const Grid* g, int f, int i, int j, int k) {
  if (f <= RIGHT) return j + g->ny * k;
  if (f <= TOP) return i + g->nx * k;
  return i + g->nx * j;
}

/* Neumann/Robin closure of one node: cpu_utils.cpp:640-717 (2D), 785-899 (3D).
 * Returns 0 when the node keeps its value (|denominator| <= 1e-12). */
static inline int nr_value(const Grid* g, int f, int loc, double u_nb, double* out) {
  const int kind = face_kind(g, f);
  const int is_max = (f & 1);
  const double h = f <= RIGHT ? g->dx : (f <= TOP ? g->dy : g->dz);
  if (kind == PDEB200_BC_NEUMANN) {
    const double gv = g->val[f][loc];
    *out = is_max ? u_nb + h * gv : u_nb - h * gv;
    return 1;
  }
  if (kind == PDEB200_BC_ROBIN) {
    const double alpha = g->al[f][loc], beta = g->be[f][loc], gamma = g->ga[f][loc];
    if (!is_max) {
      const double denom = alpha + beta / h;
      if (fabs(denom) > 1e-12) {
        *out = (gamma + (beta / h) * u_nb) / denom;
        return 1;
      }
    } else {
      const double denom = alpha - beta / h;
      if (fabs(denom) > 1e-12) {
        *out = (gamma - (beta / h) * u_nb) / denom;
        return 1;
      }
    }
  }
  return 0;
}

/* ApplyNeumannRobinCPU / ApplyNeumannRobinCPU3D: x faces, then y faces, then z faces. */
static void apply_nr(const Grid* g, double* u) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  for (int f = LEFT; f <= RIGHT; ++f) {
    if (face_kind(g, f) == PDEB200_BC_DIRICHLET) continue;
    const int i = f == LEFT ? 0 : nx - 1, inb = f == LEFT ? 1 : nx - 2;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        double v;
        if (nr_value(g, f, flocal(g, f, i, j, k), u[ID(g, inb, j, k)], &v)) u[ID(g, i, j, k)] = v;
      }
  }
  for (int f = BOTTOM; f <= TOP; ++f) {
    if (face_kind(g, f) == PDEB200_BC_DIRICHLET) continue;
    const int j = f == BOTTOM ? 0 : ny - 1, jnb = f == BOTTOM ? 1 : ny - 2;
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nx; ++i) {
        double v;
        if (nr_value(g, f, flocal(g, f, i, j, k), u[ID(g, i, jnb, k)], &v)) u[ID(g, i, j, k)] = v;
      }
  }
  if (g->dim == 3) {
    for (int f = FRONT; f <= BACK; ++f) {
      if (face_kind(g, f) == PDEB200_BC_DIRICHLET) continue;
      const int k = f == FRONT ? 0 : nz - 1, knb = f == FRONT ? 1 : nz - 2;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          double v;
          if (nr_value(g, f, flocal(g, f, i, j, k), u[ID(g, i, j, knb)], &v)) u[ID(g, i, j, k)] = v;
        }
    }
  }
}

/* ApplyDirichletCPU / ApplyDirichletCPU3D: x faces, y faces, z faces, later faces win. */
static void apply_dirichlet(const Grid* g, double* u) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      if (face_kind(g, LEFT) == PDEB200_BC_DIRICHLET) u[ID(g, 0, j, k)] = g->val[LEFT][flocal(g, LEFT, 0, j, k)];
      if (face_kind(g, RIGHT) == PDEB200_BC_DIRICHLET)
        u[ID(g, nx - 1, j, k)] = g->val[RIGHT][flocal(g, RIGHT, nx - 1, j, k)];
    }
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      if (face_kind(g, BOTTOM) == PDEB200_BC_DIRICHLET) u[ID(g, i, 0, k)] = g->val[BOTTOM][flocal(g, BOTTOM, i, 0, k)];
      if (face_kind(g, TOP) == PDEB200_BC_DIRICHLET)
        u[ID(g, i, ny - 1, k)] = g->val[TOP][flocal(g, TOP, i, ny - 1, k)];
    }
  if (g->dim == 3) {
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        if (face_kind(g, FRONT) == PDEB200_BC_DIRICHLET) u[ID(g, i, j, 0)] = g->val[FRONT][flocal(g, FRONT, i, j, 0)];
        if (face_kind(g, BACK) == PDEB200_BC_DIRICHLET)
          u[ID(g, i, j, nz - 1)] = g->val[BACK][flocal(g, BACK, i, j, nz - 1)];
      }
  }
}

static int all_dirichlet(const Grid* g) {
  for (int f = 0; f < 6; ++f)
    if (face_active(g, f) && face_kind(g, f) != PDEB200_BC_DIRICHLET) return 0;
  return 1;
}

/* ---------------------------------------------------------- relaxation */

/* One interior point update; returns the new value. Reference expression order:
 * rhs = -(f + 0 + nonlinear(old) + 0) - (lap + 0 + 0 + 0); upd = rhs/center
 * (relaxation.cpp:534-536, solver.cpp:955-962). */
static inline double relax_point(const Grid* g, const double* u, int i, int j, int k, long id) {
  Stencil s;
  node_stencil(g, i, j, k, &s);
  const double lap = nb_sum(g, &s, u, id);
  const double rhs = -(f_nl(g, id, u[id])) - (lap);
  return rhs / s.c;
}

/* SolveJacobi2D (relaxation.cpp:310-574), SolveGaussSeidelSor2D (:52-308),
 * 3D sweep (solver.cpp:749-981). */
static int relax(const Grid* g, const pdeb200_options* o, double* out, pdeb200_report* rep) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const int jacobi = o->method == PDEB200_JACOBI;
  const double omega = o->method == PDEB200_SOR ? o->sor_omega : 1.0;
  if (o->method == PDEB200_SOR && (omega <= 0.0 || omega >= 2.0)) {
    set_msg(rep, "SOR omega must be in (0,2)");
    return PDEB200_ERR_INVALID;
  }
  const int max_iter = o->max_iter > 1 ? o->max_iter : 1;
  double* grid = (double*)calloc((size_t)g->n, sizeof(double));
  double* next = jacobi ? (double*)calloc((size_t)g->n, sizeof(double)) : NULL;
  apply_dirichlet(g, grid);
  if (g->dim == 3) {
    apply_nr(g, grid);
    apply_dirichlet(g, grid);
  }
  const int k0 = g->dim == 3 ? 1 : 0, k1 = g->dim == 3 ? nz - 1 : 1;
  int iter = 0, status = PDEB200_OK;
  double max_delta = 0.0;
  for (iter = 0; iter < max_iter; ++iter) {
    if (o->cancel && *o->cancel) {
      status = PDEB200_ERR_CANCELLED;
      break;
    }
    apply_nr(g, grid);
    max_delta = 0.0;
    int degenerate = 0;
    if (jacobi) {
#pragma omp parallel for collapse(2) reduction(max : max_delta) reduction(|| : degenerate) schedule(static)
      for (int k = k0; k < k1; ++k)
        for (int j = 1; j < ny - 1; ++j)
          for (int i = 1; i < nx - 1; ++i) {
            const long id = ID(g, i, j, k);
            Stencil s;
            node_stencil(g, i, j, k, &s);
            if (fabs(s.c) < 1e-12) {
              degenerate = 1;
              continue;
            }
            const double old_u = grid[id];
            const double upd = relax_point(g, grid, i, j, k, id);
            next[id] = upd;
            const double dlt = fabs(upd - old_u);
            if (dlt > max_delta) max_delta = dlt;
          }
    } else {
      for (int k = k0; k < k1; ++k)
        for (int j = 1; j < ny - 1; ++j)
          for (int i = 1; i < nx - 1; ++i) {
            const long id = ID(g, i, j, k);
            Stencil s;
            node_stencil(g, i, j, k, &s);
            if (fabs(s.c) < 1e-12) {
              degenerate = 1;
              continue;
            }
            const double old_u = grid[id];
            const double upd = relax_point(g, grid, i, j, k, id);
            const double updated = (1.0 - omega) * old_u + omega * upd;
            grid[id] = updated;
            const double dlt = fabs(updated - old_u);
            if (dlt > max_delta) max_delta = dlt;
          }
    }
    if (degenerate) {
      status = PDEB200_ERR_DEGENERATE;
      break;
    }
    if (jacobi) {
      apply_nr(g, next);
      apply_dirichlet(g, next);
      double* t = grid;
      grid = next;
      next = t;
    } else if (g->dim == 3) {
      apply_nr(g, grid);
      apply_dirichlet(g, grid);
    }
    if (max_delta < o->tol) {
      ++iter;
      break;
    }
  }
  memcpy(out, grid, sizeof(double) * (size_t)g->n);
  free(grid);
  free(next);
  if (rep) {
    rep->iterations = iter;
    rep->last_delta = max_delta;
    rep->converged = max_delta < o->tol;
  }
  return status;
}

/* ------------------------------------------------------ operator (full) */

/* LinearOperator2D::Apply (cpu_utils.cpp:324-513): interior rows
 * center*u + neighbours, boundary rows identity; extended to 3D. */
static void apply_full(const Grid* g, const double* x, double* y) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const int k0 = g->dim == 3 ? 1 : 0, k1 = g->dim == 3 ? nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long id = ID(g, i, j, k);
        const int interior = i > 0 && i < nx - 1 && j > 0 && j < ny - 1 && k >= k0 && k < k1;
        if (!interior) {
          y[id] = x[id];
          continue;
        }
        Stencil s;
        node_stencil(g, i, j, k, &s);
        y[id] = s.c * x[id] + nb_sum(g, &s, x, id);
      }
}

static double dot(const double* a, const double* b, long n) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static double norm2(const double* a, long n) {
  const double d = dot(a, a, n);
  return sqrt(d > 0.0 ? d : 0.0);
}

/* BuildRhs2D (solver.cpp:167-232): Dirichlet values on the boundary, -f inside. */
static void build_rhs_full(const Grid* g, double* b) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  double* bnd = (double*)calloc((size_t)g->n, sizeof(double));
  apply_dirichlet(g, bnd);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long id = ID(g, i, j, k);
        const int bd = i == 0 || i == nx - 1 || j == 0 || j == ny - 1 ||
                       (g->dim == 3 && (k == 0 || k == nz - 1));
        b[id] = bd ? bnd[id] : -f_at(g, id);
      }
  free(bnd);
}

/* --------------------------------------------------------- Krylov (ref) */

typedef void (*ApplyFn)(const Grid*, const double*, double*);

/* CgSolve (krylov.cpp:14-80): x0 = 0, absolute |r| < tol on the recursive residual. */
static int cg_ref(const Grid* g, ApplyFn A, const double* b, double* x, int max_iter, double tol,
                  int relative, int* iters) {
  const long n = g->n;
  double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n);
  memset(x, 0, sizeof(double) * n);
  A(g, x, Ap);
  for (long i = 0; i < n; ++i) {
    r[i] = b[i] - Ap[i];
    p[i] = r[i];
  }
  const double scale = relative ? norm2(b, n) : 1.0;
  double rr = dot(r, r, n);
  int st = PDEB200_ERR_NOT_CONVERGED, it = 0;
  if (sqrt(rr) < tol * scale) {
    st = PDEB200_OK;
    goto done;
  }
  for (it = 0; it < max_iter; ++it) {
    A(g, p, Ap);
    const double pAp = dot(p, Ap, n);
    if (fabs(pAp) < 1e-30) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    const double alpha = rr / pAp;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    const double rr_new = dot(r, r, n);
    if (sqrt(rr_new) < tol * scale) {
      st = PDEB200_OK;
      ++it;
      break;
    }
    const double beta = rr_new / rr;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    rr = rr_new;
  }
done:
  *iters = it;
  free(r);
  free(p);
  free(Ap);
  return st;
}

/* BiCGStabSolve (krylov.cpp:82-185): true residual recomputed each iteration,
 * s-norm early exit. */
static int bicgstab_ref(const Grid* g, ApplyFn A, const double* b, double* x, int max_iter,
                        double tol, int* iters) {
  const long n = g->n;
  double* buf = calloc((size_t)n * 7, sizeof(double));
  double *r = buf, *rhat = buf + n, *p = buf + 2 * n, *v = buf + 3 * n, *s = buf + 4 * n,
         *t = buf + 5 * n, *Ax = buf + 6 * n;
  memset(x, 0, sizeof(double) * n);
  A(g, x, Ax);
  for (long i = 0; i < n; ++i) {
    r[i] = b[i] - Ax[i];
    rhat[i] = r[i];
  }
  double rho_prev = 1.0, alpha = 1.0, omega = 1.0;
  int st = PDEB200_ERR_NOT_CONVERGED, it = 0;
  if (norm2(r, n) < tol) {
    st = PDEB200_OK;
    goto done;
  }
  for (it = 0; it < max_iter; ++it) {
    const double rho = dot(rhat, r, n);
    if (fabs(rho) < 1e-30) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    if (it == 0) {
      memcpy(p, r, sizeof(double) * n);
    } else {
      const double beta = (rho / rho_prev) * (alpha / omega);
      for (long i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    }
    A(g, p, v);
    const double denom = dot(rhat, v, n);
    if (fabs(denom) < 1e-30) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    alpha = rho / denom;
    for (long i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    if (norm2(s, n) < tol) {
      for (long i = 0; i < n; ++i) x[i] += alpha * p[i];
      st = PDEB200_OK;
      ++it;
      break;
    }
    A(g, s, t);
    const double tt = dot(t, t, n);
    if (fabs(tt) < 1e-30) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    omega = dot(t, s, n) / tt;
    for (long i = 0; i < n; ++i) x[i] += alpha * p[i] + omega * s[i];
    A(g, x, Ax);
    for (long i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    if (norm2(r, n) < tol) {
      st = PDEB200_OK;
      ++it;
      break;
    }
    if (fabs(omega) < 1e-30) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    rho_prev = rho;
  }
done:
  *iters = it;
  free(buf);
  return st;
}

/* GmresSolve (krylov.cpp:187-333): GMRES(m), modified Gram-Schmidt, Givens,
 * absolute tol on |g|. The reference sizes the back-substitution with
 * y_dim = min(m, iter_total) (:297); restated as is. */
static int gmres_ref(const Grid* g, ApplyFn A, const double* b, double* x, int max_iter, int restart,
                     double tol, int* iters) {
  const long n = g->n;
  restart = restart > 1 ? restart : 1;
  max_iter = max_iter > 1 ? max_iter : 1;
  double *Ax = malloc(sizeof(double) * n), *r = malloc(sizeof(double) * n), *w = malloc(sizeof(double) * n);
  memset(x, 0, sizeof(double) * n);
  A(g, x, Ax);
  for (long i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
  double beta = norm2(r, n);
  int st = PDEB200_ERR_NOT_CONVERGED, iter_total = 0;
  if (beta < tol) {
    st = PDEB200_OK;
    goto done;
  }
  while (iter_total < max_iter) {
    const int m = restart < max_iter - iter_total ? restart : max_iter - iter_total;
    double* V = calloc((size_t)(m + 1) * n, sizeof(double));
    double* H = calloc((size_t)(m + 1) * m, sizeof(double));
    double* cs = calloc(m, sizeof(double));
    double* sn = calloc(m, sizeof(double));
    double* gv = calloc(m + 1, sizeof(double));
    double* y = calloc(m + 1, sizeof(double));
#define HH(a, bb) H[(size_t)(a) * m + (bb)]
    gv[0] = beta;
    for (long i = 0; i < n; ++i) V[i] = r[i] / beta;
    int fail = 0;
    for (int j = 0; j < m; ++j) {
      A(g, V + (size_t)j * n, w);
      for (int i = 0; i <= j; ++i) {
        HH(i, j) = dot(w, V + (size_t)i * n, n);
        const double h = HH(i, j);
        const double* vi = V + (size_t)i * n;
        for (long q = 0; q < n; ++q) w[q] -= h * vi[q];
      }
      HH(j + 1, j) = norm2(w, n);
      if (HH(j + 1, j) > 0.0) {
        double* vj = V + (size_t)(j + 1) * n;
        const double h = HH(j + 1, j);
        for (long q = 0; q < n; ++q) vj[q] = w[q] / h;
      }
      for (int i = 0; i < j; ++i) {
        const double v1 = HH(i, j), v2 = HH(i + 1, j);
        HH(i, j) = cs[i] * v1 - sn[i] * v2;
        HH(i + 1, j) = sn[i] * v1 + cs[i] * v2;
      }
      const double h_j1j = HH(j + 1, j), h_jj = HH(j, j);
      const double denom = sqrt(h_jj * h_jj + h_j1j * h_j1j);
      if (denom < 1e-30) {
        fail = 1;
        break;
      }
      cs[j] = h_jj / denom;
      sn[j] = -h_j1j / denom;
      HH(j, j) = cs[j] * h_jj - sn[j] * h_j1j;
      HH(j + 1, j) = 0.0;
      const double g1 = gv[j], g2 = gv[j + 1];
      gv[j] = cs[j] * g1 - sn[j] * g2;
      gv[j + 1] = sn[j] * g1 + cs[j] * g2;
      ++iter_total;
      if (fabs(gv[j + 1]) < tol) break;
    }
    if (!fail) {
      const int y_dim = m < iter_total ? m : iter_total;
      for (int i = y_dim - 1; i >= 0; --i) {
        double sum = gv[i];
        for (int kk = i + 1; kk < y_dim; ++kk) sum -= HH(i, kk) * y[kk];
        if (fabs(HH(i, i)) < 1e-30) {
          fail = 1;
          break;
        }
        y[i] = sum / HH(i, i);
      }
      if (!fail)
        for (int j = 0; j < y_dim; ++j) {
          const double* vj = V + (size_t)j * n;
          for (long q = 0; q < n; ++q) x[q] += y[j] * vj[q];
        }
    }
#undef HH
    free(V);
    free(H);
    free(cs);
    free(sn);
    free(gv);
    free(y);
    if (fail) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    A(g, x, Ax);
    for (long i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    beta = norm2(r, n);
    if (beta < tol) {
      st = PDEB200_OK;
      break;
    }
    if (iter_total >= max_iter) break;
  }
done:
  *iters = iter_total;
  free(Ax);
  free(r);
  free(w);
  return st;
}

/* ------------------------------------------------ MG V-cycle (reference) */

/* MultigridVcyclePoisson (multigrid.cpp:121-222): one V-cycle, lexicographic
 * GS, constant a,b,e, coarsen while odd >= 5, coarsest at n <= 5. */
typedef struct {
  int nx, ny;
  double dx, dy;
  double *u, *b, *r;
} MgLevel2;

static void mg2_coeffs(const MgLevel2* L, double a, double bc, double e, double* ax, double* by,
                       double* center) {
  *ax = a / (L->dx * L->dx);
  *by = bc / (L->dy * L->dy);
  *center = -2.0 * (*ax) - 2.0 * (*by) + e;
}

static void mg2_smooth(MgLevel2* L, double ax, double by, double center, int iters) {
  const int nx = L->nx, ny = L->ny;
  for (int it = 0; it < iters; ++it)
    for (int j = 1; j < ny - 1; ++j)
      for (int i = 1; i < nx - 1; ++i) {
        const long id = (long)j * nx + i;
        const double rhs = L->b[id] - ax * (L->u[id - 1] + L->u[id + 1]) - by * (L->u[id - nx] + L->u[id + nx]);
        L->u[id] = rhs / center;
      }
}

static int mg_vcycle_ref(const Grid* g, const pdeb200_options* o, const double* b, double* u) {
  const pdeb200_problem* p = g->p;
  if (!(g->nx >= 5 && g->nx % 2 == 1 && g->ny >= 5 && g->ny % 2 == 1)) return PDEB200_ERR_UNSUPPORTED;
  int max_levels = o->mg_max_levels;
  MgLevel2 lv[32];
  int L = 0;
  lv[0].nx = g->nx;
  lv[0].ny = g->ny;
  lv[0].dx = (p->xmax - p->xmin) / (double)(g->nx - 1);
  lv[0].dy = (p->ymax - p->ymin) / (double)(g->ny - 1);
  lv[0].u = malloc(sizeof(double) * g->n);
  memcpy(lv[0].u, u, sizeof(double) * g->n);
  lv[0].b = malloc(sizeof(double) * g->n);
  memcpy(lv[0].b, b, sizeof(double) * g->n);
  lv[0].r = calloc(g->n, sizeof(double));
  L = 1;
  while (L < max_levels && L < 32) {
    const MgLevel2* pr = &lv[L - 1];
    if (!(pr->nx >= 5 && pr->nx % 2 == 1 && pr->ny >= 5 && pr->ny % 2 == 1)) break;
    const int ncx = (pr->nx + 1) / 2, ncy = (pr->ny + 1) / 2;
    if (ncx < 3 || ncy < 3) break;
    MgLevel2* c = &lv[L];
    c->nx = ncx;
    c->ny = ncy;
    c->dx = (p->xmax - p->xmin) / (double)(ncx - 1);
    c->dy = (p->ymax - p->ymin) / (double)(ncy - 1);
    c->u = calloc((size_t)ncx * ncy, sizeof(double));
    c->b = calloc((size_t)ncx * ncy, sizeof(double));
    c->r = calloc((size_t)ncx * ncy, sizeof(double));
    ++L;
    if (ncx <= 5 || ncy <= 5) break;
  }
  int st = PDEB200_OK;
  for (int l = 0; l < L - 1 && st == PDEB200_OK; ++l) {
    double ax, by, center;
    mg2_coeffs(&lv[l], p->a, p->b, p->e, &ax, &by, &center);
    if (fabs(center) < 1e-12) {
      st = PDEB200_ERR_DEGENERATE;
      break;
    }
    mg2_smooth(&lv[l], ax, by, center, o->mg_pre_smooth > 0 ? o->mg_pre_smooth : 0);
    /* ResidualPoisson (multigrid.cpp:96-119) */
    MgLevel2* F = &lv[l];
    memset(F->r, 0, sizeof(double) * (size_t)F->nx * F->ny);
    for (int j = 1; j < F->ny - 1; ++j)
      for (int i = 1; i < F->nx - 1; ++i) {
        const long id = (long)j * F->nx + i;
        const double Au = center * F->u[id] + ax * (F->u[id - 1] + F->u[id + 1]) +
                          by * (F->u[id - F->nx] + F->u[id + F->nx]);
        F->r[id] = F->b[id] - Au;
      }
    /* RestrictFullWeighting (multigrid.cpp:14-36) */
    MgLevel2* Cc = &lv[l + 1];
    memset(Cc->b, 0, sizeof(double) * (size_t)Cc->nx * Cc->ny);
    for (int jc = 1; jc < Cc->ny - 1; ++jc)
      for (int ic = 1; ic < Cc->nx - 1; ++ic) {
        const int ifx = 2 * ic, jf = 2 * jc, fx = F->nx;
        const double* fr = F->r;
        const double c = fr[(long)jf * fx + ifx] * 0.25;
        const double e = (fr[(long)jf * fx + ifx - 1] + fr[(long)jf * fx + ifx + 1] +
                          fr[(long)(jf - 1) * fx + ifx] + fr[(long)(jf + 1) * fx + ifx]) * 0.125;
        const double d = (fr[(long)(jf - 1) * fx + ifx - 1] + fr[(long)(jf - 1) * fx + ifx + 1] +
                          fr[(long)(jf + 1) * fx + ifx - 1] + fr[(long)(jf + 1) * fx + ifx + 1]) * 0.0625;
        Cc->b[(long)jc * Cc->nx + ic] = c + e + d;
      }
    memset(Cc->u, 0, sizeof(double) * (size_t)Cc->nx * Cc->ny);
  }
  if (st == PDEB200_OK) {
    double ax, by, center;
    mg2_coeffs(&lv[L - 1], p->a, p->b, p->e, &ax, &by, &center);
    if (fabs(center) < 1e-12)
      st = PDEB200_ERR_DEGENERATE;
    else
      mg2_smooth(&lv[L - 1], ax, by, center, o->mg_coarse_iters > 1 ? o->mg_coarse_iters : 1);
  }
  for (int l = L - 2; l >= 0 && st == PDEB200_OK; --l) {
    MgLevel2 *F = &lv[l], *Cc = &lv[l + 1];
    /* ProlongBilinearAdd (multigrid.cpp:38-67) */
    for (int jc = 0; jc < Cc->ny; ++jc)
      for (int ic = 0; ic < Cc->nx; ++ic) {
        const double vc = Cc->u[(long)jc * Cc->nx + ic];
        const int ifx = 2 * ic, jf = 2 * jc, fx = F->nx;
        if (ifx < F->nx && jf < F->ny) F->u[(long)jf * fx + ifx] += vc;
        if (ic + 1 < Cc->nx && ifx + 1 < F->nx && jf < F->ny) {
          const double vr = Cc->u[(long)jc * Cc->nx + ic + 1];
          F->u[(long)jf * fx + ifx + 1] += 0.5 * (vc + vr);
        }
        if (jc + 1 < Cc->ny && ifx < F->nx && jf + 1 < F->ny) {
          const double vu = Cc->u[(long)(jc + 1) * Cc->nx + ic];
          F->u[(long)(jf + 1) * fx + ifx] += 0.5 * (vc + vu);
        }
        if (ic + 1 < Cc->nx && jc + 1 < Cc->ny && ifx + 1 < F->nx && jf + 1 < F->ny) {
          const double vru = Cc->u[(long)(jc + 1) * Cc->nx + ic + 1];
          const double vr = Cc->u[(long)jc * Cc->nx + ic + 1];
          const double vu = Cc->u[(long)(jc + 1) * Cc->nx + ic];
          F->u[(long)(jf + 1) * fx + ifx + 1] += 0.25 * (vc + vr + vu + vru);
        }
      }
    double ax, by, center;
    mg2_coeffs(F, p->a, p->b, p->e, &ax, &by, &center);
    if (fabs(center) < 1e-12) {
      st = PDEB200_ERR_DEGENERATE;
      break;
    }
    mg2_smooth(F, ax, by, center, o->mg_post_smooth > 0 ? o->mg_post_smooth : 0);
  }
  if (st == PDEB200_OK) memcpy(u, lv[0].u, sizeof(double) * g->n);
  for (int l = 0; l < L; ++l) {
    free(lv[l].u);
    free(lv[l].b);
    free(lv[l].r);
  }
  return st;
}

/* ------------------------------------------------------- folded system */

/* The B200 Krylov/MG forms solve for the interior nodes only; every boundary
 * node is eliminated through its closure u_b = c0 + c1*u_nb (the closure the
 * reference relaxation applies each iteration, cpu_utils.cpp:630-901), which
 * leaves a symmetric operator for symmetric stencils:
 *   diag  = center + w_face*c1,   b = -f - w_face*c0.
 * Dirichlet: c0 = value, c1 = 0. Neumann: c0 = -+h*g, c1 = 1.
 * Robin min face: c0 = gamma/(alpha+beta/h), c1 = (beta/h)/(alpha+beta/h);
 * max face: c0 = gamma/(alpha-beta/h), c1 = -(beta/h)/(alpha-beta/h). */
static void face_c01(const Grid* g, int f, int loc, double* c0, double* c1) {
  const int kind = face_kind(g, f);
  const int is_max = f & 1;
  const double h = f <= RIGHT ? g->dx : (f <= TOP ? g->dy : g->dz);
  if (kind == PDEB200_BC_DIRICHLET) {
    *c0 = g->val[f][loc];
    *c1 = 0.0;
  } else if (kind == PDEB200_BC_NEUMANN) {
    *c0 = is_max ? h * g->val[f][loc] : -h * g->val[f][loc];
    *c1 = 1.0;
  } else {
    const double bh = g->be[f][loc] / h;
    const double den = is_max ? g->al[f][loc] - bh : g->al[f][loc] + bh;
    *c0 = g->ga[f][loc] / den;
    *c1 = (is_max ? -bh : bh) / den;
  }
}

/* Folded stencil of interior node (i,j,k): face-neighbour weights moved into the
 * diagonal (and their c0 part returned in *bshift, to subtract from -f). */
static void folded_stencil(const Grid* g, int i, int j, int k, Stencil* s, double* bshift) {
  node_stencil(g, i, j, k, s);
  double shift = 0.0, c0, c1;
  if (i == 1) { face_c01(g, LEFT, flocal(g, LEFT, 0, j, k), &c0, &c1); s->c += s->xm * c1; shift += s->xm * c0; s->xm = 0.0; }
  if (i == g->nx - 2) { face_c01(g, RIGHT, flocal(g, RIGHT, g->nx - 1, j, k), &c0, &c1); s->c += s->xp * c1; shift += s->xp * c0; s->xp = 0.0; }
  if (j == 1) { face_c01(g, BOTTOM, flocal(g, BOTTOM, i, 0, k), &c0, &c1); s->c += s->ym * c1; shift += s->ym * c0; s->ym = 0.0; }
  if (j == g->ny - 2) { face_c01(g, TOP, flocal(g, TOP, i, g->ny - 1, k), &c0, &c1); s->c += s->yp * c1; shift += s->yp * c0; s->yp = 0.0; }
  if (g->dim == 3) {
    if (k == 1) { face_c01(g, FRONT, flocal(g, FRONT, i, j, 0), &c0, &c1); s->c += s->zm * c1; shift += s->zm * c0; s->zm = 0.0; }
    if (k == g->nz - 2) { face_c01(g, BACK, flocal(g, BACK, i, j, g->nz - 1), &c0, &c1); s->c += s->zp * c1; shift += s->zp * c0; s->zp = 0.0; }
  }
  if (bshift) *bshift = shift;
}

static inline int is_interior(const Grid* g, int i, int j, int k) {
  if (i <= 0 || i >= g->nx - 1 || j <= 0 || j >= g->ny - 1) return 0;
  if (g->dim == 3 && (k <= 0 || k >= g->nz - 1)) return 0;
  return 1;
}

static void folded_rhs(const Grid* g, double* b) {
  memset(b, 0, sizeof(double) * g->n);
  const int k0 = g->dim == 3 ? 1 : 0, k1 = g->dim == 3 ? g->nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < k1; ++k)
    for (int j = 1; j < g->ny - 1; ++j)
      for (int i = 1; i < g->nx - 1; ++i) {
        Stencil s;
        double sh;
        folded_stencil(g, i, j, k, &s, &sh);
        const long id = ID(g, i, j, k);
        b[id] = -f_at(g, id) - sh;
      }
}

static void folded_apply(const Grid* g, const double* x, double* y) {
  memset(y, 0, sizeof(double) * g->n);
  const int k0 = g->dim == 3 ? 1 : 0, k1 = g->dim == 3 ? g->nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < k1; ++k)
    for (int j = 1; j < g->ny - 1; ++j)
      for (int i = 1; i < g->nx - 1; ++i) {
        Stencil s;
        folded_stencil(g, i, j, k, &s, NULL);
        const long id = ID(g, i, j, k);
        y[id] = s.c * x[id] + nb_sum(g, &s, x, id);
      }
}

/* Boundary of a field from its interior: Dirichlet, Neumann/Robin (x, y, z
 * faces), Dirichlet — the sequence of solver.cpp:751-753. */
static void fill_boundary(const Grid* g, double* u) {
  apply_dirichlet(g, u);
  apply_nr(g, u);
  apply_dirichlet(g, u);
}

/* ---------------------------------------------------- MG hierarchy (B200) */

/* Geometric hierarchy of the folded operator: vertex-centred coarsening
 * n_c = ceil((n-1)/2) + 1 per dimension (coarse_dims; for odd cubes the 2:1
 * coarsening of multigrid.cpp:150-170, continued down to 3 nodes; even n gives
 * non-nested levels), coarse k from the nearest fine
 * node, faces sampled at the nearest finest-level face node, h rediscretised. */
typedef struct {
  Grid g;
  pdeb200_problem p;
  double* k;      /* DIVK coefficient of this level (owned for l > 0) */
  double *x, *b, *r;
} Level;

static int coarse_size(int n) { return n / 2 + 1; } /* ceil((n-1)/2) + 1 */

/* Per-dimension coarsening: a dimension with >= 5 nodes coarsens when its
 * spacing is below twice the smallest spacing (semi-coarsening on elongated
 * grids); 0 when none does. */
static int coarse_dims(const Grid* g, int nc[3]) {
  const int n[3] = {g->nx, g->ny, g->nz};
  const double h[3] = {g->dx, g->dy, g->dz};
  const int dims = g->dim == 3 ? 3 : 2;
  double hmin = h[0];
  int any = 0;
  for (int d = 1; d < dims; ++d)
    if (h[d] < hmin) hmin = h[d];
  for (int d = 0; d < 3; ++d) {
    nc[d] = n[d];
    if (d < dims && n[d] >= 5 && h[d] < 2.0 * hmin) {
      nc[d] = coarse_size(n[d]);
      any = 1;
    }
  }
  return any;
}

/* nearest fine node of coarse node I (coarse I sits at I*(n-1)/(nc-1)) */
static int nearest_fine(int I, int n, int nc) {
  if (nc <= 1) return 0;
  return (I * (n - 1) + (nc - 1) / 2) / (nc - 1);
}

static int build_levels(const Grid* g0, int max_levels, Level* lv) {
  int L = 0;
  lv[0].g = *g0;
  lv[0].p = *g0->p;
  lv[0].g.p = &lv[0].p;
  lv[0].k = (double*)g0->p->k;
  L = 1;
  while (L < max_levels && L < 16) {
    const Grid* pg = &lv[L - 1].g;
    int nc[3];
    if (!coarse_dims(pg, nc)) break;
    Level* c = &lv[L];
    c->p = lv[L - 1].p;
    c->p.nx = nc[0];
    c->p.ny = nc[1];
    c->p.nz = pg->dim == 3 ? nc[2] : 1;
    /* coarse faces: constants only (per-node face arrays are sampled below) */
    for (int f = 0; f < 6; ++f) {
      c->p.face[f].value_arr = c->p.face[f].alpha_arr = c->p.face[f].beta_arr = c->p.face[f].gamma_arr = NULL;
    }
    if (grid_init(&c->g, &c->p) != PDEB200_OK) break;
    for (int f = 0; f < 6; ++f) {
      const Grid* fg = &lv[0].g;
      const int w = f <= RIGHT ? c->g.ny : c->g.nx;
      const int h = f <= RIGHT ? c->g.nz : (f <= TOP ? c->g.nz : c->g.ny);
      const int fw = f <= RIGHT ? fg->ny : fg->nx;
      const int fh = f <= RIGHT ? fg->nz : (f <= TOP ? fg->nz : fg->ny);
      for (int q = 0; q < c->g.fsize[f]; ++q) {
        /* face parameters: coarse face node (a,b) <- nearest finest face node */
        const int qa = q % w, qb = q / w;
        const int fq = nearest_fine(qa, fw, w) + fw * nearest_fine(qb, fh, h);
        c->g.val[f][q] = fg->val[f][fq];
        c->g.al[f][q] = fg->al[f][fq];
        c->g.be[f][q] = fg->be[f][fq];
        c->g.ga[f][q] = fg->ga[f][fq];
      }
    }
    c->g.p = &c->p;
    c->k = NULL;
    if (c->p.coef_kind == PDEB200_COEF_DIVK) {
      c->k = malloc(sizeof(double) * c->g.n);
      for (int k = 0; k < c->g.nz; ++k)
        for (int j = 0; j < c->g.ny; ++j)
          for (int i = 0; i < c->g.nx; ++i)
            c->k[ID(&c->g, i, j, k)] =
                lv[L - 1].k[ID(pg, nearest_fine(i, pg->nx, c->g.nx), nearest_fine(j, pg->ny, c->g.ny),
                               pg->dim == 3 ? nearest_fine(k, pg->nz, c->g.nz) : 0)];
      c->p.k = c->k;
    }
    c->p.f = NULL;
    ++L;
  }
  for (int l = 0; l < L; ++l) {
    lv[l].x = calloc(lv[l].g.n, sizeof(double));
    lv[l].b = calloc(lv[l].g.n, sizeof(double));
    lv[l].r = calloc(lv[l].g.n, sizeof(double));
  }
  return L;
}

/* Interpolation position of fine node i: coarse interval I0 and weight t of
 * node I0+1 (exact rational position i*(nc-1)/(n-1)). */
static void coarse_pos(int i, int n, int nc, int* I0, double* t) {
  const int num = i * (nc - 1);
  *I0 = num / (n - 1);
  *t = (double)(num - *I0 * (n - 1)) / (double)(n - 1);
  if (*I0 >= nc - 1) {
    *I0 = nc - 1;
    *t = 0.0;
  }
}

/* Restriction weights (scaled transpose of the interpolation) of coarse node
 * I: w_i = (nc-1)/(n-1) * max(0, 1 - |i(nc-1) - I(n-1)|/(n-1)). */
static int restrict_weights(int I, int n, int nc, int* idx, double* w) {
  const int den = n - 1;
  const double scale = (double)(nc - 1) / (double)den;
  int cnt = 0;
  for (int i = 0; i < n; ++i) {
    int d = i * (nc - 1) - I * den;
    if (d < 0) d = -d;
    if (d < den) {
      idx[cnt] = i;
      w[cnt] = scale * (1.0 - (double)d / (double)den);
      ++cnt;
    }
  }
  return cnt;
}

static void free_levels(Level* lv, int L) {
  for (int l = 0; l < L; ++l) {
    free(lv[l].x);
    free(lv[l].b);
    free(lv[l].r);
    if (l > 0) {
      free(lv[l].k);
      grid_free(&lv[l].g);
    }
  }
}

/* One red-black Gauss-Seidel colour pass on the folded operator; colour =
 * (i+j+k) & 1. */
static void rbgs_color(const Grid* g, const double* b, double* x, int color) {
  const int k0 = g->dim == 3 ? 1 : 0, k1 = g->dim == 3 ? g->nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < k1; ++k)
    for (int j = 1; j < g->ny - 1; ++j)
      for (int i = 1 + ((1 + j + k + color) & 1); i < g->nx - 1; i += 2) {
        Stencil s;
        folded_stencil(g, i, j, k, &s, NULL);
        const long id = ID(g, i, j, k);
        x[id] = (b[id] - nb_sum(g, &s, x, id)) / s.c;
      }
}

/* Visit the nodes of face f in (k, j, i) order with i, j, k in scope. Within
 * one face pass no two nodes share an inward neighbour, so the order of the
 * visits does not change any value. */
#define FACE_NODES(g, f, ...)                                                      \
  do {                                                                             \
    const int k_lo_ = (f) == BACK ? (g)->nz - 1 : 0, k_hi_ = (f) == FRONT ? 1 : (g)->nz; \
    const int j_lo_ = (f) == TOP ? (g)->ny - 1 : 0, j_hi_ = (f) == BOTTOM ? 1 : (g)->ny; \
    const int i_lo_ = (f) == RIGHT ? (g)->nx - 1 : 0, i_hi_ = (f) == LEFT ? 1 : (g)->nx; \
    for (int k = k_lo_; k < k_hi_; ++k)                                            \
      for (int j = j_lo_; j < j_hi_; ++j)                                          \
        for (int i = i_lo_; i < i_hi_; ++i) __VA_ARGS__                            \
  } while (0)

/* The interior neighbour of face node (i, j, k) across face f. */
static inline void inward(const Grid* g, int f, int i, int j, int k, int* ii, int* jj, int* kk) {
  *ii = f == LEFT ? 1 : f == RIGHT ? g->nx - 2 : i;
  *jj = f == BOTTOM ? 1 : f == TOP ? g->ny - 2 : j;
  *kk = f == FRONT ? 1 : f == BACK ? g->nz - 2 : k;
}

/* Homogeneous closure extension of a correction field: boundary nodes take
 * c1 * (inward neighbour) in the reference's phase order (x, y, z faces),
 * Dirichlet nodes 0. Ext is the map the folded system eliminates, so
 * interpolating Ext(x_c) carries Neumann/Robin corrections to the faces. */
static void ext_apply(const Grid* g, double* x) {
  double c0, c1;
  for (int f = LEFT; f <= BACK; ++f) {
    if (!face_active(g, f) || face_kind(g, f) != PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, x[ID(g, i, j, k)] = 0.0;);
  }
  for (int f = LEFT; f <= BACK; ++f) {
    if (!face_active(g, f) || face_kind(g, f) == PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, {
      int ii, jj, kk;
      inward(g, f, i, j, k, &ii, &jj, &kk);
      face_c01(g, f, flocal(g, f, i, j, k), &c0, &c1);
      x[ID(g, i, j, k)] = c1 * x[ID(g, ii, jj, kk)];
    });
  }
  for (int f = LEFT; f <= BACK; ++f) {
    if (!face_active(g, f) || face_kind(g, f) != PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, x[ID(g, i, j, k)] = 0.0;);
  }
}

/* Transpose of ext_apply: Dirichlet nodes zeroed, then the Neumann/Robin
 * phases in reverse (z, y, x): y[inward] += c1*y[b], y[b] = 0. */
static void ext_transpose(const Grid* g, double* y) {
  double c0, c1;
  for (int f = LEFT; f <= BACK; ++f) {
    if (!face_active(g, f) || face_kind(g, f) != PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, y[ID(g, i, j, k)] = 0.0;);
  }
  for (int f = BACK; f >= LEFT; --f) {
    if (!face_active(g, f) || face_kind(g, f) == PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, {
      int ii, jj, kk;
      inward(g, f, i, j, k, &ii, &jj, &kk);
      face_c01(g, f, flocal(g, f, i, j, k), &c0, &c1);
      y[ID(g, ii, jj, kk)] += c1 * y[ID(g, i, j, k)];
      y[ID(g, i, j, k)] = 0.0;
    });
  }
  for (int f = LEFT; f <= BACK; ++f) {
    if (!face_active(g, f) || face_kind(g, f) != PDEB200_BC_DIRICHLET) continue;
    FACE_NODES(g, f, y[ID(g, i, j, k)] = 0.0;);
  }
}

static int g_mg_boundary_transfer = 1;
void rs_set_mg_boundary_transfer(int on) { g_mg_boundary_transfer = on; }

static void mg_vcycle_folded(Level* lv, int L, int l, int pre, int post, int coarse_iters) {
  Grid* g = &lv[l].g;
  double *x = lv[l].x, *b = lv[l].b;
  memset(x, 0, sizeof(double) * g->n);
  if (l == L - 1) {
    for (int it = 0; it < coarse_iters; ++it) {
      rbgs_color(g, b, x, 0);
      rbgs_color(g, b, x, 1);
    }
    return;
  }
  for (int it = 0; it < pre; ++it) {
    rbgs_color(g, b, x, 0);
    rbgs_color(g, b, x, 1);
  }
  /* r = b - A x */
  folded_apply(g, x, lv[l].r);
#pragma omp parallel for schedule(static)
  for (long q = 0; q < g->n; ++q) lv[l].r[q] = b[q] - lv[l].r[q];
  /* full weighting r -> coarse b (tensor [1/4,1/2,1/4] for odd n, the scaled
   * transpose of the interpolation in general) at every coarse node, then the
   * transpose of the boundary extension
   * folds the boundary-node values into the interior: R = Ext^T P^T / 2^dim. */
  Grid* c = &lv[l + 1].g;
  double* bc = lv[l + 1].b;
  memset(bc, 0, sizeof(double) * c->n);
  const int all = g_mg_boundary_transfer;
  const int kc0 = c->dim == 3 ? (all ? 0 : 1) : 0, kc1 = c->dim == 3 ? (all ? c->nz : c->nz - 1) : 1;
  const int ic0 = all ? 0 : 1, ic1 = all ? c->nx : c->nx - 1, jc0 = all ? 0 : 1, jc1 = all ? c->ny : c->ny - 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int K = kc0; K < kc1; ++K)
    for (int J = jc0; J < jc1; ++J)
      for (int I = ic0; I < ic1; ++I) {
        int ix[4], iy[4], iz[4];
        double wx[4], wy[4], wz[4];
        const int nxw = restrict_weights(I, g->nx, c->nx, ix, wx);
        const int nyw = restrict_weights(J, g->ny, c->ny, iy, wy);
        int nzw = 1;
        if (c->dim == 3) {
          nzw = restrict_weights(K, g->nz, c->nz, iz, wz);
        } else {
          iz[0] = 0;
          wz[0] = 1.0;
        }
        double acc = 0.0;
        for (int cc = 0; cc < nzw; ++cc)
          for (int bb = 0; bb < nyw; ++bb) {
            double rs = 0.0;
            for (int aa = 0; aa < nxw; ++aa) rs += wx[aa] * lv[l].r[ID(g, ix[aa], iy[bb], iz[cc])];
            acc += wz[cc] * wy[bb] * rs;
          }
        bc[ID(c, I, J, K)] = acc;
      }
  if (all) ext_transpose(c, bc);
  mg_vcycle_folded(lv, L, l + 1, pre, post, coarse_iters);
  /* trilinear prolongation-add of the coarse correction, extended to the
   * coarse boundary by the homogeneous closures */
  double* xc = lv[l + 1].x;
  if (g_mg_boundary_transfer) ext_apply(c, xc);
  const int kf0 = g->dim == 3 ? 1 : 0, kf1 = g->dim == 3 ? g->nz - 1 : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = kf0; k < kf1; ++k)
    for (int j = 1; j < g->ny - 1; ++j)
      for (int i = 1; i < g->nx - 1; ++i) {
        int I0, J0, K0 = 0;
        double tx, ty, tz = 0.0;
        coarse_pos(i, g->nx, c->nx, &I0, &tx);
        coarse_pos(j, g->ny, c->ny, &J0, &ty);
        if (g->dim == 3) coarse_pos(k, g->nz, c->nz, &K0, &tz);
        const int I1 = I0 + 1 < c->nx ? I0 + 1 : c->nx - 1, J1 = J0 + 1 < c->ny ? J0 + 1 : c->ny - 1;
        const int K1 = g->dim == 3 ? (K0 + 1 < c->nz ? K0 + 1 : c->nz - 1) : 0;
        const double x00 = (1.0 - tx) * xc[ID(c, I0, J0, K0)] + tx * xc[ID(c, I1, J0, K0)];
        const double x10 = (1.0 - tx) * xc[ID(c, I0, J1, K0)] + tx * xc[ID(c, I1, J1, K0)];
        const double x01 = (1.0 - tx) * xc[ID(c, I0, J0, K1)] + tx * xc[ID(c, I1, J0, K1)];
        const double x11 = (1.0 - tx) * xc[ID(c, I0, J1, K1)] + tx * xc[ID(c, I1, J1, K1)];
        const double y0 = (1.0 - ty) * x00 + ty * x10, y1 = (1.0 - ty) * x01 + ty * x11;
        const double v = (1.0 - tz) * y0 + tz * y1;
        x[ID(g, i, j, k)] += v;
      }
  for (int it = 0; it < post; ++it) {
    rbgs_color(g, b, x, 1);
    rbgs_color(g, b, x, 0);
  }
}

/* MG-preconditioned CG on the folded system (the B200 MG_PCG form), relative
 * tolerance on the recursive residual, confirmed on the true residual. */
static int mg_pcg(const Grid* g, const pdeb200_options* o, double* x, pdeb200_report* rep) {
  Level lv[16];
  const int L = build_levels(g, o->mg_max_levels > 0 ? o->mg_max_levels : 1, lv);
  const long n = g->n;
  double* b = malloc(sizeof(double) * n);
  double* r = malloc(sizeof(double) * n);
  double* z = malloc(sizeof(double) * n);
  double* p = malloc(sizeof(double) * n);
  double* q = malloc(sizeof(double) * n);
  folded_rhs(g, b);
  memset(x, 0, sizeof(double) * n);
  memcpy(r, b, sizeof(double) * n);
  const double bnorm = norm2(b, n);
  int st = PDEB200_ERR_NOT_CONVERGED, it = 0;
  double rr = dot(r, r, n);
  if (bnorm == 0.0 || sqrt(rr) <= o->tol * bnorm) {
    st = PDEB200_OK;
    goto finish;
  }
#define PRECOND(dst)                                                         \
  do {                                                                       \
    memcpy(lv[0].b, r, sizeof(double) * n);                                  \
    memset(lv[0].x, 0, sizeof(double) * n);                                  \
    mg_vcycle_folded(lv, L, 0, o->mg_pre_smooth, o->mg_post_smooth, o->mg_coarse_iters); \
    memcpy(dst, lv[0].x, sizeof(double) * n);                                \
  } while (0)
  PRECOND(z);
  memcpy(p, z, sizeof(double) * n);
  double rz = dot(r, z, n);
  for (it = 0; it < o->max_iter; ++it) {
    folded_apply(g, p, q);
    const double pq = dot(p, q, n);
    if (fabs(pq) < 1e-300) {
      st = PDEB200_ERR_BREAKDOWN;
      break;
    }
    const double alpha = rz / pq;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rr = dot(r, r, n);
    if (sqrt(rr) <= o->tol * bnorm) {
      st = PDEB200_OK;
      ++it;
      break;
    }
    PRECOND(z);
    const double rz_new = dot(r, z, n);
    const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
#undef PRECOND
finish:
  folded_apply(g, x, q);
  for (long i = 0; i < n; ++i) q[i] = b[i] - q[i];
  if (rep) {
    rep->iterations = it;
    rep->residual_l2 = norm2(q, n);
    rep->rhs_l2 = bnorm;
    rep->rel_residual = bnorm > 0 ? rep->residual_l2 / bnorm : 0.0;
    rep->converged = st == PDEB200_OK;
  }
  fill_boundary(g, x);
  free(b);
  free(r);
  free(z);
  free(p);
  free(q);
  free_levels(lv, L);
  return st;
}

/* -------------------------------------------------------------- entries */

void rs_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

int rs_solve(const pdeb200_problem* prob, const pdeb200_options* o, double* out, pdeb200_report* rep) {
  Grid g;
  if (rep) memset(rep, 0, sizeof(*rep));
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) {
    set_msg(rep, "invalid grid");
    return st;
  }
  st = check_center(&g);
  if (st != PDEB200_OK) {
    set_msg(rep, "degenerate PDE center coefficient");
    grid_free(&g);
    return st;
  }
  double omp0 = omp_get_wtime();
  if (prob->n_nonlinear > 0 && o->method != PDEB200_JACOBI && o->method != PDEB200_GAUSS_SEIDEL &&
      o->method != PDEB200_SOR) {
    /* solver.cpp:502,550 */
    set_msg(rep, o->method >= PDEB200_CG && o->method <= PDEB200_GMRES ? "Krylov solvers require linear PDEs"
                                                                      : "Multigrid requires linear PDEs");
    grid_free(&g);
    return PDEB200_ERR_UNSUPPORTED;
  }
  switch (o->method) {
    case PDEB200_JACOBI:
    case PDEB200_GAUSS_SEIDEL:
    case PDEB200_SOR:
      st = relax(&g, o, out, rep);
      break;
    case PDEB200_CG:
    case PDEB200_BICGSTAB:
    case PDEB200_GMRES: {
      if (!all_dirichlet(&g)) {
        set_msg(rep, "Krylov solvers require Dirichlet boundaries on all sides");
        st = PDEB200_ERR_UNSUPPORTED;
        break;
      }
      double* b = malloc(sizeof(double) * g.n);
      build_rhs_full(&g, b);
      int it = 0;
      const int rel = o->tol_mode == PDEB200_TOL_RELATIVE;
      if (o->method == PDEB200_CG)
        st = cg_ref(&g, apply_full, b, out, o->max_iter > 1 ? o->max_iter : 1, o->tol, rel, &it);
      else if (o->method == PDEB200_BICGSTAB)
        st = bicgstab_ref(&g, apply_full, b, out, o->max_iter > 1 ? o->max_iter : 1, o->tol, &it);
      else
        st = gmres_ref(&g, apply_full, b, out, o->max_iter, o->gmres_restart, o->tol, &it);
      if (rep) {
        double* t = malloc(sizeof(double) * g.n);
        apply_full(&g, out, t);
        for (long i = 0; i < g.n; ++i) t[i] = b[i] - t[i];
        rep->iterations = it;
        rep->residual_l2 = norm2(t, g.n);
        rep->rhs_l2 = norm2(b, g.n);
        rep->rel_residual = rep->rhs_l2 > 0 ? rep->residual_l2 / rep->rhs_l2 : 0.0;
        rep->converged = st == PDEB200_OK;
        free(t);
      }
      free(b);
      break;
    }
    case PDEB200_MG_VCYCLE: {
      if (g.dim != 2 || !all_dirichlet(&g) || prob->coef_kind != PDEB200_COEF_CONST ||
          fabs(prob->c) > 1e-12 || fabs(prob->d) > 1e-12) {
        set_msg(rep, "reference multigrid: 2D, Dirichlet, constant a,b,e only");
        st = PDEB200_ERR_UNSUPPORTED;
        break;
      }
      double* b = malloc(sizeof(double) * g.n);
      build_rhs_full(&g, b);
      memset(out, 0, sizeof(double) * g.n);
      apply_dirichlet(&g, out);
      st = mg_vcycle_ref(&g, o, b, out);
      if (rep) rep->iterations = 1;
      free(b);
      break;
    }
    case PDEB200_MG_PCG:
      st = mg_pcg(&g, o, out, rep);
      break;
    default:
      st = PDEB200_ERR_UNSUPPORTED;
  }
  if (rep) rep->total_ms = 1e3 * (omp_get_wtime() - omp0);
  grid_free(&g);
  return st;
}

int rs_apply(const pdeb200_problem* prob, const double* x, double* y) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  apply_full(&g, x, y);
  grid_free(&g);
  return PDEB200_OK;
}

int rs_folded_rhs(const pdeb200_problem* prob, double* b) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  folded_rhs(&g, b);
  grid_free(&g);
  return PDEB200_OK;
}

int rs_folded_apply(const pdeb200_problem* prob, const double* x, double* y) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  folded_apply(&g, x, y);
  grid_free(&g);
  return PDEB200_OK;
}

int rs_fill_boundary(const pdeb200_problem* prob, double* grid) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  fill_boundary(&g, grid);
  grid_free(&g);
  return PDEB200_OK;
}

/* ComputeResidualNorms (src/residual.cpp:153-723). 2D: every node, boundary
 * nodes by their closure with alpha + beta/h on all Robin faces (:359,399);
 * 3D: interior only. Kahan-summed squares (:51-60). */
int rs_residual_norms(const pdeb200_problem* prob, const double* grid, double* l2, double* linf) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  double sum = 0.0, comp = 0.0, mx = 0.0;
#define ACC(rv)                              \
  do {                                       \
    const double rr_ = (rv);                 \
    const double yv = rr_ * rr_ - comp;      \
    const double tv = sum + yv;              \
    comp = (tv - sum) - yv;                  \
    sum = tv;                                \
    if (fabs(rr_) > mx) mx = fabs(rr_);      \
  } while (0)
  const int nx = g.nx, ny = g.ny;
  if (g.dim == 2) {
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const long id = ID(&g, i, j, 0);
        const double u = grid[id];
        int f = -1, nb = -1;
        double h = 0.0;
        if (i == 0) { f = LEFT; nb = (int)ID(&g, 1, j, 0); h = g.dx; }
        else if (i == nx - 1) { f = RIGHT; nb = (int)ID(&g, nx - 2, j, 0); h = g.dx; }
        else if (j == 0) { f = BOTTOM; nb = (int)ID(&g, i, 1, 0); h = g.dy; }
        else if (j == ny - 1) { f = TOP; nb = (int)ID(&g, i, ny - 2, 0); h = g.dy; }
        if (f >= 0) {
          const int loc = flocal(&g, f, i, j, 0);
          const int kind = face_kind(&g, f);
          if (kind == PDEB200_BC_DIRICHLET) {
            ACC(u - g.val[f][loc]);
          } else if (kind == PDEB200_BC_NEUMANN) {
            const double gv = g.val[f][loc];
            const double target = (f & 1) ? grid[nb] + h * gv : grid[nb] - h * gv;
            ACC(u - target);
          } else {
            const double alpha = g.al[f][loc], beta = g.be[f][loc], gamma = g.ga[f][loc];
            const double denom = alpha + beta / h;
            if (fabs(denom) > 1e-12) {
              const double target = (gamma + (beta / h) * grid[nb]) / denom;
              ACC(u - target);
            }
          }
          continue;
        }
        Stencil s;
        node_stencil(&g, i, j, 0, &s);
        const double r = s.c * u + nb_sum(&g, &s, grid, id) + (f_nl(&g, id, u));
        ACC(r);
      }
  } else {
    for (int k = 1; k < g.nz - 1; ++k)
      for (int j = 1; j < ny - 1; ++j)
        for (int i = 1; i < nx - 1; ++i) {
          const long id = ID(&g, i, j, k);
          Stencil s;
          node_stencil(&g, i, j, k, &s);
          const double r = s.c * grid[id] + nb_sum(&g, &s, grid, id) + f_at(&g, id);
          ACC(r);
        }
  }
#undef ACC
  *l2 = sqrt(sum > 0 ? sum : 0.0);
  *linf = mx;
  grid_free(&g);
  return PDEB200_OK;
}

/* SolvePDETimeSeries forward Euler (solver.cpp:1244-1324), one step per frame:
 * u+ = u + dt * SafeDivClamped(-(L u + f), ut, 0) in the interior, then
 * Neumann/Robin and Dirichlet closures; 3D uses the 7-point stencil and the
 * 3D closures (the reference's 3D series is a stub, solver.cpp:1331-1334). */
int rs_time_series(const pdeb200_problem* prob, const pdeb200_time_options* t, double* out,
                   double* frames_out) {
  Grid g;
  int st = grid_init(&g, prob);
  if (st != PDEB200_OK) return st;
  if (t->dt <= 0.0) {
    grid_free(&g);
    return PDEB200_ERR_INVALID;
  }
  const long n = g.n;
  double* grid = calloc(n, sizeof(double));
  double* next = calloc(n, sizeof(double));
  double* opv = calloc(n, sizeof(double));
  if (prob->u0) memcpy(grid, prob->u0, sizeof(double) * n);
  apply_dirichlet(&g, grid);
  apply_nr(&g, grid);
  apply_dirichlet(&g, grid);
  const int frames = t->frames > 1 ? t->frames : 1;
  const double ut = prob->ut;
  const int k0 = g.dim == 3 ? 1 : 0, k1 = g.dim == 3 ? g.nz - 1 : 1;
  for (int frame = 0; frame < frames; ++frame) {
    if (frames_out) memcpy(frames_out + (size_t)frame * n, grid, sizeof(double) * n);
    if (frame + 1 >= frames) break;
    apply_full(&g, grid, opv);
    memcpy(next, grid, sizeof(double) * n);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = k0; k < k1; ++k)
      for (int j = 1; j < g.ny - 1; ++j)
        for (int i = 1; i < g.nx - 1; ++i) {
          const long id = ID(&g, i, j, k);
          const double rhs = g.p->n_nonlinear ? opv[id] + f_at(&g, id) + eval_nonlinear(g.p, grid[id])
                                              : opv[id] + f_at(&g, id);
          double u_t = 0.0;
          if (fabs(ut) >= 1e-12) {
            u_t = -rhs / ut;
            if (!isfinite(u_t)) u_t = 0.0;
          }
          next[id] = grid[id] + t->dt * u_t;
        }
    double* tmp = grid;
    grid = next;
    next = tmp;
    apply_nr(&g, grid);
    apply_dirichlet(&g, grid);
  }
  memcpy(out, grid, sizeof(double) * n);
  free(grid);
  free(next);
  free(opv);
  grid_free(&g);
  return PDEB200_OK;
}

/* ProjectVelocity2D / 3D (pressure_projection.cpp:255-334, 694-761):
 * collocated central divergence (one-sided at walls), pure-Neumann pressure
 * Poisson by CG with mean projection (2D, :111-249) or a pinned corner (3D,
 * :504-692), gradient update. */
int rs_project(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double* u,
               double* v, double* w, double* pres, const pdeb200_projection_options* po,
               pdeb200_projection_report* rep) {
  const int is3 = nz > 1;
  const int NZ = is3 ? nz : 1;
  const long n = (long)nx * ny * NZ, sxy = (long)nx * ny;
  double* div = malloc(sizeof(double) * n);
#define DIVERGENCE()                                                                          \
  for (int k = 0; k < NZ; ++k)                                                                \
    for (int j = 0; j < ny; ++j)                                                              \
      for (int i = 0; i < nx; ++i) {                                                          \
        const long id = k * sxy + (long)j * nx + i;                                           \
        double du, dv, dw = 0.0;                                                              \
        if (i == 0) du = (u[id + 1] - u[id]) / dx;                                            \
        else if (i == nx - 1) du = (u[id] - u[id - 1]) / dx;                                  \
        else du = (u[id + 1] - u[id - 1]) / (2.0 * dx);                                       \
        if (j == 0) dv = (v[id + nx] - v[id]) / dy;                                           \
        else if (j == ny - 1) dv = (v[id] - v[id - nx]) / dy;                                 \
        else dv = (v[id + nx] - v[id - nx]) / (2.0 * dy);                                     \
        if (is3) {                                                                            \
          if (k == 0) dw = (w[id + sxy] - w[id]) / dz;                                        \
          else if (k == NZ - 1) dw = (w[id] - w[id - sxy]) / dz;                              \
          else dw = (w[id + sxy] - w[id - sxy]) / (2.0 * dz);                                 \
          div[id] = du + dv + dw;                                                             \
        } else {                                                                              \
          div[id] = du + dv;                                                                  \
        }                                                                                     \
      }
  DIVERGENCE();
  double l2b = 0.0, mxb = 0.0;
  for (long i = 0; i < n; ++i) {
    l2b += div[i] * div[i];
    if (fabs(div[i]) > mxb) mxb = fabs(div[i]);
  }
  rep->l2_divergence_before = sqrt(l2b / n);
  rep->max_divergence_before = mxb;
  double* rhs = malloc(sizeof(double) * n);
  for (long i = 0; i < n; ++i) rhs[i] = div[i] / dt;
  /* SolvePressurePoisson */
  const double cx = 1.0 / (dx * dx), cy = 1.0 / (dy * dy), cz = is3 ? 1.0 / (dz * dz) : 0.0;
  const double cc = is3 ? -2.0 * (cx + cy + cz) : 0.0;
  double mean = 0.0;
  for (long i = 0; i < n; ++i) mean += rhs[i];
  mean /= n;
  for (long i = 0; i < n; ++i) rhs[i] -= mean;
  const int pin = is3 && po->fix_pressure_corner;
  if (pin) rhs[0] = po->reference_pressure;
  double *r = calloc(n, sizeof(double)), *pc = calloc(n, sizeof(double)), *Ap = calloc(n, sizeof(double));
#define LAPLACE(X, Y)                                                                     \
  for (int k = 0; k < NZ; ++k)                                                            \
    for (int j = 0; j < ny; ++j)                                                          \
      for (int i = 0; i < nx; ++i) {                                                      \
        const long id = k * sxy + (long)j * nx + i;                                       \
        const double xc = X[id];                                                          \
        if (!is3) {                                                                       \
          const double xm = i > 0 ? X[id - 1] : xc, xp = i < nx - 1 ? X[id + 1] : xc;     \
          const double ym = j > 0 ? X[id - nx] : xc, yp = j < ny - 1 ? X[id + nx] : xc;   \
          Y[id] = cx * (xp - 2.0 * xc + xm) + cy * (yp - 2.0 * xc + ym);                  \
        } else {                                                                          \
          double lap = cc * xc;                                                           \
          lap += cx * (i > 0 ? X[id - 1] : xc);                                           \
          lap += cx * (i < nx - 1 ? X[id + 1] : xc);                                      \
          lap += cy * (j > 0 ? X[id - nx] : xc);                                          \
          lap += cy * (j < ny - 1 ? X[id + nx] : xc);                                     \
          lap += cz * (k > 0 ? X[id - sxy] : xc);                                         \
          lap += cz * (k < NZ - 1 ? X[id + sxy] : xc);                                    \
          Y[id] = lap;                                                                    \
        }                                                                                 \
      }                                                                                   \
  if (pin) Y[0] = X[0];
  LAPLACE(pres, Ap);
  for (long i = 0; i < n; ++i) r[i] = rhs[i] - Ap[i];
  if (!is3) {
    double mr = 0.0;
    for (long i = 0; i < n; ++i) mr += r[i];
    mr /= n;
    for (long i = 0; i < n; ++i) r[i] -= mr;
  }
  memcpy(pc, r, sizeof(double) * n);
  double rr = 0.0;
  for (long i = 0; i < n; ++i) rr += r[i] * r[i];
  const double r0 = sqrt(rr);
  int ok = 1, iters = 0, done = 0;
  double resid = 0.0;
  if (r0 < 1e-15) {
    done = 1;
    iters = 0;
    resid = 0.0;
  }
  for (int it = 0; !done && it < po->max_iter; ++it) {
    LAPLACE(pc, Ap);
    if (!is3) {
      double ma = 0.0;
      for (long i = 0; i < n; ++i) ma += Ap[i];
      ma /= n;
      for (long i = 0; i < n; ++i) Ap[i] -= ma;
    }
    double pAp = 0.0;
    for (long i = 0; i < n; ++i) pAp += pc[i] * Ap[i];
    if (fabs(pAp) < 1e-30) {
      iters = it;
      resid = sqrt(rr);
      ok = !is3;
      done = 1;
      break;
    }
    const double alpha = rr / pAp;
    for (long i = 0; i < n; ++i) {
      pres[i] += alpha * pc[i];
      r[i] -= alpha * Ap[i];
    }
    double rn = 0.0;
    for (long i = 0; i < n; ++i) rn += r[i] * r[i];
    const double rnorm = sqrt(rn);
    if (rnorm < po->tol * r0 || rnorm < 1e-14) {
      iters = it + 1;
      resid = rnorm;
      double mp = 0.0;
      for (long i = 0; i < n; ++i) mp += pres[i];
      mp /= n;
      for (long i = 0; i < n; ++i) pres[i] -= mp;
      done = 2;
      break;
    }
    const double beta = rn / rr;
    for (long i = 0; i < n; ++i) pc[i] = r[i] + beta * pc[i];
    rr = rn;
  }
  if (!done) {
    if (!is3) {
      double mp = 0.0;
      for (long i = 0; i < n; ++i) mp += pres[i];
      mp /= n;
      for (long i = 0; i < n; ++i) pres[i] -= mp;
    } else {
      ok = 0;
    }
    iters = po->max_iter;
    resid = sqrt(rr);
  }
#undef LAPLACE
  rep->poisson_iterations = iters;
  rep->poisson_residual = resid;
  if (ok) {
    for (int k = 0; k < NZ; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const long id = k * sxy + (long)j * nx + i;
          double gx, gy, gz = 0.0;
          if (i == 0) gx = (pres[id + 1] - pres[id]) / dx;
          else if (i == nx - 1) gx = (pres[id] - pres[id - 1]) / dx;
          else gx = (pres[id + 1] - pres[id - 1]) / (2.0 * dx);
          if (j == 0) gy = (pres[id + nx] - pres[id]) / dy;
          else if (j == ny - 1) gy = (pres[id] - pres[id - nx]) / dy;
          else gy = (pres[id + nx] - pres[id - nx]) / (2.0 * dy);
          if (is3) {
            if (k == 0) gz = (pres[id + sxy] - pres[id]) / dz;
            else if (k == NZ - 1) gz = (pres[id] - pres[id - sxy]) / dz;
            else gz = (pres[id + sxy] - pres[id - sxy]) / (2.0 * dz);
          }
          div[id] = gx;  /* reuse buffers: gx in div, gy in Ap, gz in r */
          Ap[id] = gy;
          r[id] = gz;
        }
    for (long i = 0; i < n; ++i) {
      u[i] -= dt * div[i];
      v[i] -= dt * Ap[i];
      if (is3) w[i] -= dt * r[i];
    }
    DIVERGENCE();
    double l2a = 0.0, mxa = 0.0;
    for (long i = 0; i < n; ++i) {
      l2a += div[i] * div[i];
      if (fabs(div[i]) > mxa) mxa = fabs(div[i]);
    }
    rep->l2_divergence_after = sqrt(l2a / n);
    rep->max_divergence_after = mxa;
  }
#undef DIVERGENCE
  rep->success = ok;
  free(div);
  free(rhs);
  free(r);
  free(pc);
  free(Ap);
  return ok ? PDEB200_OK : PDEB200_ERR_NOT_CONVERGED;
}

/* sizeof of the ABI structs as compiled by a C compiler from include/pdeb200.h
 * (tests compare them with the ctypes mirror). */
long rs_sizeof(int which) {
  switch (which) {
    case 0: return (long)sizeof(pdeb200_face);
    case 1: return (long)sizeof(pdeb200_problem);
    case 2: return (long)sizeof(pdeb200_options);
    case 3: return (long)sizeof(pdeb200_report);
    case 4: return (long)sizeof(pdeb200_time_options);
    case 5: return (long)sizeof(pdeb200_projection_options);
    case 6: return (long)sizeof(pdeb200_projection_report);
    case 7: return (long)sizeof(pdeb200_batch_options);
    case 8: return (long)sizeof(pdeb200_batch_stats);
    case 9: return (long)sizeof(pdeb200_server_options);
    case 10: return (long)sizeof(pdeb200_request);
    case 11: return (long)sizeof(pdeb200_result);
    case 12: return (long)sizeof(pdeb200_server_stats);
    default: return -1;
  }
}
