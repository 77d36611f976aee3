/*
 * pdeb200.h — C ABI of the B200 structured-grid solve library (libpdeb200.so).
 *
 * This is the boundary that replaces the reference's CUDA backend
 * (pde_solver: include/cuda_solver.h:8-9, src/backends/cuda/CudaSolve.h:7-10).
 * The C++ shim pde_solver_b200/shim/cuda_solver_shim.cpp implements the
 * reference signatures `bool CudaIsAvailable(std::string*)` and
 * `SolveOutput SolvePDECuda(const SolveInput&)` on top of these entry points;
 * any other host (ctypes, cgo, JNI) binds the same symbols directly.
 *
 * Conventions (all follow the reference CPU solver):
 *   - node-centred uniform grid, x_i = xmin + i*dx, dx = (xmax-xmin)/(nx-1)
 *     (src/backends/cpu/solver.cpp:462-467, include/safe_math.h:155-157);
 *   - flat index (k*ny + j)*nx + i, x fastest (src/backends/cpu/cpu_utils.h:13-19);
 *   - discrete equation  sum(coeff * D(u)) + f = 0 with
 *     center = -2a/dx^2 - 2b/dy^2 - 2az/dz^2 + e (src/backends/cpu/solver.cpp:723-729),
 *     so -Laplace(u) = F is a = b = az = -1, f = -F;
 *   - face order left(x=xmin), right(x=xmax), bottom(y=ymin), top(y=ymax),
 *     front(z=zmin), back(z=zmax) (include/pde_types.h:192-199);
 *   - all arithmetic of the plain path is IEEE FP64.
 *
 * Errors: every entry point returns a pdeb200_status; no exceptions cross the
 * ABI. pdeb200_status_string() gives the text the shim copies into
 * SolveOutput.error (the reference reports errors as strings, include/pde_types.h:417).
 *
 * Threading: calls are synchronous and blocking on the caller's thread, like
 * the reference entry (src/backend_solve.cpp:166-179). Device memory is owned
 * by the library; a per-device context caches workspaces between calls, so
 * repeated solves of one shape allocate nothing after the first.
 */
#ifndef PDEB200_H
#define PDEB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDEB200_ABI_VERSION 2

typedef enum {
  PDEB200_OK = 0,
  PDEB200_ERR_INVALID = 1,        /* bad sizes, bounds, null pointers */
  PDEB200_ERR_UNSUPPORTED = 2,    /* method/feature combination not offered */
  PDEB200_ERR_NO_DEVICE = 3,      /* no CUDA device / library built without one */
  PDEB200_ERR_CUDA = 4,           /* CUDA runtime error (message in report) */
  PDEB200_ERR_OOM = 5,            /* device memory (or admission budget) exhausted */
  PDEB200_ERR_NOT_CONVERGED = 6,  /* iteration cap reached (result still written) */
  PDEB200_ERR_BREAKDOWN = 7,      /* Krylov breakdown (|denominator| < 1e-30) */
  PDEB200_ERR_DEGENERATE = 8,     /* |center| < 1e-12 somewhere */
  PDEB200_ERR_CANCELLED = 9,      /* cancel flag observed */
  PDEB200_ERR_TIMEOUT = 10,       /* a bounded device wait expired */
  PDEB200_ERR_BUSY = 11           /* server queue full */
} pdeb200_status;

/* Boundary kinds, same order as BCKind (include/pde_types.h:172-179). */
typedef enum {
  PDEB200_BC_DIRICHLET = 0,
  PDEB200_BC_NEUMANN = 1,
  PDEB200_BC_ROBIN = 2
} pdeb200_bc_kind;

/* One face. Constant parts are used where the matching array is NULL.
 * Arrays are indexed by the face-local node index:
 *   left/right  : j + ny*k      (ny*nz entries)
 *   bottom/top  : i + nx*k      (nx*nz entries)
 *   front/back  : i + nx*j      (nx*ny entries)
 * Closures (src/backends/cpu/cpu_utils.cpp:630-720, 774-901):
 *   Dirichlet  u_b = value
 *   Neumann    u_0 = u_1 - h*value (min face), u_N = u_{N-1} + h*value (max face)
 *   Robin      u_0 = (gamma + beta/h*u_1)/(alpha + beta/h)         (min face)
 *              u_N = (gamma - beta/h*u_{N-1})/(alpha - beta/h)     (max face)
 */
typedef struct {
  int32_t kind;
  int32_t reserved;
  double value;
  double alpha;
  double beta;
  double gamma;
  const double* value_arr;
  const double* alpha_arr;
  const double* beta_arr;
  const double* gamma_arr;
} pdeb200_face;

/* Coefficient forms of the operator. */
typedef enum {
  /* constant a,b,az,c,d,dz,e: the reference's Cartesian FD stencil
   * (src/backends/cpu/cpu_utils.cpp:421-433, src/backends/cpu/solver.cpp:892-898) */
  PDEB200_COEF_CONST = 0,
  /* divergence form with a node-sampled diffusivity k:
   *   L u = sum_faces (k_face/h^2)(u_i - u_nb) + convection(c,d,dz) + e*u,
   *   k_face = (k_i + k_nb)/2.  Constant k is exactly a=b=az=-k. */
  PDEB200_COEF_DIVK = 1,
  /* per-node a,b,az,c,d,dz,e arrays (7*N doubles, array-major): the reference's
   * variable-coefficient non-divergence stencil (src/backends/cpu/solver.cpp:838-898) */
  PDEB200_COEF_NODAL = 2
} pdeb200_coef_kind;

/* Pointwise nonlinear terms sum(coeff * g(u)) of the discrete equation
 * (NonlinearTerm / NonlinearKind, include/pde_types.h:88-100), evaluated at
 * the node's current value the way EvalNonlinear does
 * (src/backends/cpu/solvers/relaxation.cpp:27-45, src/backends/cpu/solver.cpp:234-256):
 * g = u^power, sin u, cos u, exp u or |u|. The relaxation methods (Jacobi,
 * Gauss-Seidel, SOR), the explicit time series and the residual norms take
 * them; the Krylov and multigrid methods reject them, as the reference does
 * (src/backends/cpu/solver.cpp:502,550). */
#define PDEB200_MAX_NONLINEAR 8

typedef enum {
  PDEB200_NL_POWER = 0,
  PDEB200_NL_SIN = 1,
  PDEB200_NL_COS = 2,
  PDEB200_NL_EXP = 3,
  PDEB200_NL_ABS = 4
} pdeb200_nonlinear_kind;

typedef struct {
  int32_t kind;   /* pdeb200_nonlinear_kind */
  int32_t power;  /* NL_POWER exponent */
  double coeff;
} pdeb200_nonlinear_term;

/* Where the pointers of a problem live. */
typedef enum {
  PDEB200_MEM_HOST = 0,   /* host pointers; copies are part of the call */
  PDEB200_MEM_DEVICE = 1  /* device pointers on options.device; output is a device pointer */
} pdeb200_mem_space;

typedef struct {
  int32_t nx, ny, nz;        /* nz <= 1 selects 2D */
  int32_t coef_kind;         /* pdeb200_coef_kind */
  int32_t mem_space;         /* pdeb200_mem_space for k, nodal, f, u0 and out_grid */
  int32_t reserved;
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double a, b, az, c, d, dz, e;  /* PDECoefficients (include/pde_types.h:10-17) */
  double f_const;                /* used where f == NULL */
  double ut;                     /* u_t coefficient (time stepping only) */
  const double* k;               /* COEF_DIVK diffusivity, N values */
  const double* nodal;           /* COEF_NODAL: a,b,az,c,d,dz,e arrays, 7*N values */
  const double* f;               /* per-node f in the reference sign convention, N values */
  const double* u0;              /* initial field (time series) or initial guess, N values */
  pdeb200_face face[6];
  int32_t n_nonlinear;           /* 0 .. PDEB200_MAX_NONLINEAR */
  int32_t reserved2;
  const pdeb200_nonlinear_term* nonlinear;  /* host array of n_nonlinear terms (any mem_space) */
} pdeb200_problem;

/* Methods: the first seven are SolveMethod (include/pde_types.h:230-238) with the
 * reference's semantics; the rest are the B200 forms. */
typedef enum {
  PDEB200_JACOBI = 0,
  PDEB200_GAUSS_SEIDEL = 1,
  PDEB200_SOR = 2,
  PDEB200_CG = 3,
  PDEB200_BICGSTAB = 4,
  PDEB200_GMRES = 5,
  PDEB200_MG_VCYCLE = 6,
  PDEB200_MG_PCG = 7,        /* geometric-MG V(pre,post) preconditioned CG, folded BCs */
  PDEB200_MG_BICGSTAB = 8    /* MG preconditioned BiCGStab (nonsymmetric operators) */
} pdeb200_method;

typedef enum {
  /* the method's reference stopping rule: Krylov absolute |r|_2 < tol on the
   * recursive residual (src/backends/cpu/solvers/krylov.cpp:39,66), relaxation
   * max|du| < tol (relaxation.cpp:557), "mg" exactly one V-cycle (solver.cpp:582) */
  PDEB200_TOL_REFERENCE = 0,
  /* |b - A u|_2 / |b|_2 <= tol on the (folded) system, checked on the true residual */
  PDEB200_TOL_RELATIVE = 1
} pdeb200_tol_mode;

typedef enum {
  PDEB200_FP64 = 0,
  /* FP32 MG + FP32 Krylov inside FP64 iterative refinement; BF16 smoother
   * coefficients when options.bf16_coefficients is set */
  PDEB200_MIXED = 1
} pdeb200_precision;

typedef enum {
  /* wavefront-ordered sweep that reproduces the reference's lexicographic
   * Gauss-Seidel/SOR exactly (src/backends/cpu/solvers/relaxation.cpp:167-289) */
  PDEB200_ORDER_LEXICOGRAPHIC = 0,
  PDEB200_ORDER_REDBLACK = 1
} pdeb200_ordering;

typedef struct {
  int32_t method;            /* pdeb200_method */
  int32_t max_iter;
  double tol;
  int32_t tol_mode;          /* pdeb200_tol_mode */
  int32_t precision;         /* pdeb200_precision */
  double sor_omega;          /* SolverConfig::sor_omega */
  int32_t gmres_restart;     /* SolverConfig::gmres_restart */
  int32_t mg_pre_smooth;     /* SolverConfig::mg_pre_smooth .. mg_max_levels */
  int32_t mg_post_smooth;
  int32_t mg_coarse_iters;
  int32_t mg_max_levels;
  int32_t gs_ordering;       /* pdeb200_ordering for GAUSS_SEIDEL / SOR */
  int32_t device;            /* CUDA device ordinal */
  int32_t check_interval;    /* host convergence poll period (iterations); 0 = auto */
  double inner_tol;          /* MIXED: relative tolerance of each inner FP32 solve (default 1e-5); a
                                last refinement step asks only the reduction the target needs */
  int32_t bf16_coefficients; /* MIXED: store smoother k in BF16 */
  int32_t max_outer;         /* MIXED: iterative-refinement cap */
  const volatile int32_t* cancel; /* polled between iterations (SolveInput::cancel) */
} pdeb200_options;

typedef struct {
  int32_t iterations;        /* Krylov/relaxation iterations (total inner for MIXED) */
  int32_t outer_iterations;  /* MIXED refinement steps */
  int32_t converged;
  int32_t kernel_launches;   /* kernels this call launched */
  double residual_l2;        /* final |b - A u|_2 of the solved system (true residual) */
  double rhs_l2;             /* |b|_2 of the solved system */
  double rel_residual;       /* residual_l2 / rhs_l2 */
  double last_delta;         /* relaxation: final max|du| */
  double device_ms;          /* device time of the solve (CUDA events) */
  double total_ms;           /* wall time of the call */
  char message[256];
} pdeb200_report;

/* ---- library / device ------------------------------------------------- */

/* ABI version; a binding checks it before use. */
int32_t pdeb200_abi_version(void);

/* Replaces CudaIsAvailable (src/backends/cuda/CudaSolve.cu:9-29):
 * 1 when a CUDA device is usable, note gets "device: <name>" or the reason. */
int32_t pdeb200_probe(char* note, size_t note_len);

/* Text for a status (the shim's SolveOutput.error). */
const char* pdeb200_status_string(int32_t status);

/* Default options: SolverConfig defaults (include/pde_types.h:282-303). */
void pdeb200_default_options(pdeb200_options* opt);

/* Frees every cached workspace of every device context. */
void pdeb200_release_all(void);

/* Launch stream (a cudaStream_t passed as void*) of every later call on
 * `device`; NULL restores the library's own non-blocking stream. Lets a host
 * that owns a stream (torch, a serving loop) order and time the solves on it. */
pdeb200_status pdeb200_set_stream(int32_t device, void* stream);

/* Per-kernel device-time accounting: while enabled, each finest-level launch
 * of the hot kernels is bracketed by CUDA events on its launch stream. */
typedef struct {
  char name[48];
  int64_t launches;
  double total_ms;          /* summed event-measured durations */
  double bytes_per_launch;  /* algorithmic bytes of one launch (finest level) */
} pdeb200_kernel_stat;

void pdeb200_profile_enable(int32_t device, int32_t on);
/* Copies up to max_stats entries; returns the number of kernels recorded. */
int32_t pdeb200_profile_read(int32_t device, pdeb200_kernel_stat* stats, int32_t max_stats);

/* ---- steady solve ----------------------------------------------------- */

/* Replaces SolvePDECuda's dispatch (src/backends/cuda/CudaSolve.cu:31-64) and
 * the three CUDA solvers (solvers/relaxation.cu:163, krylov.cu:371, multigrid.cu:287).
 * Writes the full nx*ny*nz field (boundary included) to out_grid. */
pdeb200_status pdeb200_solve(const pdeb200_problem* prob, const pdeb200_options* opt,
                             double* out_grid, pdeb200_report* report);

/* Discrete residual norms with the semantics of ComputeResidualNorms
 * (src/residual.cpp:153-723): 2D includes boundary closures (Robin uses
 * alpha + beta/h on every face, src/residual.cpp:359,399); 3D is interior only.
 * Replaces the CPU post-pass MaybeComputeResiduals (src/backend_solve.cpp:40-50). */
pdeb200_status pdeb200_residual_norms(const pdeb200_problem* prob, const double* grid,
                                      int32_t device, double* l2, double* linf);

/* One application y = L x of the full-grid operator with identity boundary rows,
 * LinearOperator2D::Apply semantics (src/backends/cpu/cpu_utils.cpp:324-513),
 * extended to 3D and to COEF_DIVK / COEF_NODAL. */
pdeb200_status pdeb200_apply(const pdeb200_problem* prob, const double* x, double* y,
                             int32_t device);

/* ---- explicit time stepping (SolvePDETimeSeries, solver.cpp:989-1329) ---- */

/* Called after each frame with the field (host pointer when the problem is
 * MEM_HOST); return 0 to stop (FrameCallback, include/solver.h:9-11). */
typedef int32_t (*pdeb200_frame_cb)(int32_t frame, double time, const double* grid,
                                    void* user);

typedef struct {
  double t_start;
  double dt;
  int32_t frames;            /* one FE step per frame (solver.cpp:1244-1264) */
  int32_t frame_stride;      /* call on_frame every n frames (1 = every frame) */
  int32_t device;
  int32_t reserved;
} pdeb200_time_options;

pdeb200_status pdeb200_time_series(const pdeb200_problem* prob, const pdeb200_time_options* topt,
                                   pdeb200_frame_cb on_frame, void* user,
                                   double* out_grid, pdeb200_report* report);

/* ---- pressure projection (src/pressure_projection.cpp:255-334, 463-761) ---- */

typedef struct {
  int32_t max_iter;          /* ProjectionConfig::max_iter */
  int32_t fix_pressure_corner; /* 3D only: pin p[0] (pressure_projection.cpp:614-621) */
  double tol;                /* relative: |r| < tol*|r0| */
  double reference_pressure;
  int32_t device;
  int32_t mem_space;         /* pdeb200_mem_space of u, v, w, pressure */
} pdeb200_projection_options;

typedef struct {
  int32_t success;
  int32_t poisson_iterations;
  double poisson_residual;
  double max_divergence_before, max_divergence_after;
  double l2_divergence_before, l2_divergence_after;
  double device_ms;
  char message[256];
} pdeb200_projection_report;

/* nz <= 1 selects 2D (w ignored). u, v, w, pressure are updated in place. */
pdeb200_status pdeb200_project_velocity(int32_t nx, int32_t ny, int32_t nz,
                                        double dx, double dy, double dz, double dt,
                                        double* u, double* v, double* w, double* pressure,
                                        const pdeb200_projection_options* popt,
                                        pdeb200_projection_report* report);

/* ---- solve without device allocation ----------------------------------- */

/* No counterpart in the reference: an addition for callers that cannot let a
 * library allocate device memory (code running inside another runtime's fixed
 * memory arena, hosts that forbid allocation after start-up). Runs the Jacobi
 * method with pdeb200_solve's semantics, but allocates nothing: the problem's
 * k / nodal / f arrays and out_grid are device pointers (mem_space DEVICE),
 * faces take constant values only, and the solver's scratch (second field,
 * reduction partials, control block) is one file-scope device array of about
 * 8.3 MB that every GPU loading the library keeps until the process exits.
 * Grids above 1048576 nodes, or with more than 8192 x-y blocks of 32 x 8
 * columns (ceil(nx/32)*ceil(ny/8) > 8192, e.g. a long, thin 2D grid), are
 * rejected (PDEB200_ERR_UNSUPPORTED). All calls share that array: calls that
 * overlap on the GPU race, so callers serialise them. Every call looks up the
 * array's address (so a device reset between calls is harmless); the first
 * call on a device also loads the module there and should come before any
 * stream capture on that device. `stream` may be NULL (the default stream). */
pdeb200_status pdeb200_jacobi_noalloc(const pdeb200_problem* prob, int32_t max_iter, double tol,
                                      int32_t device, void* stream, double* out_grid,
                                      pdeb200_report* report);

/* ---- expressions of x, y, z, t on the grid ----------------------------- */

/* Fills out[(k*ny + j)*nx + i] with the LaTeX expression evaluated at node
 * (xmin + i*dx, ymin + j*dy, zmin + k*dz) and time t, on the GPU. Replaces the
 * reference's per-node host loops over ExpressionEvaluator::Eval
 * (src/expression_eval.cpp:805-978; called per node from
 * src/backends/cpu/solver.cpp:197 for the right side and
 * src/backends/cpu/cpu_utils.cpp:520-530 for variable coefficients). Same
 * language as ExpressionEvaluator::ParseLatex: \frac, \sqrt, \cdot, \times,
 * \pi, \theta, \phi, \left/\right, \operatorname{}, the one-argument
 * functions sin ... erf (ln, arcsin, arccos, arctan, sgn as aliases), min,
 * max, atan2, pow; x/r, y/theta, z/phi, t, pi, e; implicit multiplication;
 * guarded division, powers, logarithms and roots that give NaN where the
 * reference does. Only the geometry of `grid` (nx, ny, nz, bounds) is used;
 * nz <= 1 gives z = 0. `out` is a host array of N doubles, or a device
 * pointer when mem_space is PDEB200_MEM_DEVICE. A parse error returns
 * PDEB200_ERR_INVALID with the reference's message in `message`. */
pdeb200_status pdeb200_eval_expression(const char* latex, const pdeb200_problem* grid, double t,
                                       int32_t device, double* out, int32_t mem_space,
                                       char* message, size_t message_len);

/* One boundary expression on the nodes of one face (0..5 = left, right,
 * bottom, top, front, back), in the face-local order of pdeb200_face arrays,
 * with the reference's EvalExpr rule (src/backends/cpu/cpu_utils.cpp:520-530):
 * the LaTeX value where `latex` parses and the value is finite, else the
 * linear form linear[0] + linear[1]*x + linear[2]*y + linear[3]*z
 * (BoundaryCondition::Expression, include/pde_types.h). `latex` may be NULL
 * or empty, and an expression that does not parse is not an error (the
 * linear form is used), as in the reference. `linear` may be NULL (zeros).
 * Faces 4 and 5 need nz > 1. */
pdeb200_status pdeb200_eval_face_expression(const char* latex, const double* linear,
                                            const pdeb200_problem* grid, int32_t face, double t,
                                            int32_t device, double* out, int32_t mem_space,
                                            char* message, size_t message_len);

/* The same compiled expression evaluated once on the host (no GPU), for
 * checking the compiler against ExpressionEvaluator. */
pdeb200_status pdeb200_expression_value(const char* latex, double x, double y, double z,
                                        double t, double* value, char* message,
                                        size_t message_len);

/* ---- VTK output of a grid field ----------------------------------------- */

/* Called as the write advances; fraction in [0, 1]. */
typedef void (*pdeb200_write_progress)(double fraction, void* user);

/* Legacy ASCII STRUCTURED_POINTS file, byte-identical to the reference's
 * WriteVtkStructuredPoints (src/vtk_writer.cpp:28-82): the header with the
 * ostream's default number format, then every value cast to float and printed
 * fixed with 6 decimals, followed by a space, with a newline after each x row.
 * The text is formatted on the GPU and written in chunks that overlap the
 * formatting of the next chunk. Only the geometry of `grid` is used (nz <= 1
 * writes nz = 1; the z bounds appear in ORIGIN and SPACING as given).
 * `field` holds nx*ny*nz doubles, a device pointer when mem_space is
 * PDEB200_MEM_DEVICE. Errors: PDEB200_ERR_INVALID with the reference's
 * "invalid grid dimensions" / "failed to open output file". */
pdeb200_status pdeb200_write_vtk(const char* path, const pdeb200_problem* grid, const double* field,
                                 int32_t mem_space, int32_t device, pdeb200_write_progress progress,
                                 void* user, char* message, size_t message_len);

/* XML ImageData file (.vti) with base64 Float32 arrays, byte-identical to
 * WriteVtkXmlImageData (src/vtk_writer.cpp:176-268). With `derived` set it
 * adds the derived fields of ComputeDerivedFields (src/vtk_writer.cpp:365-440)
 * in the order BuildDerivedFieldVectors lists them (src/main.cpp:255-288):
 * gradient_x, gradient_y, [gradient_z], laplacian, flux_x, flux_y, [flux_z],
 * energy_norm, with the flux coefficients grid->a, grid->b, grid->az. Each
 * array is computed and encoded on the GPU in one pass over the field. */
pdeb200_status pdeb200_write_vti(const char* path, const pdeb200_problem* grid, const double* field,
                                 int32_t derived, int32_t mem_space, int32_t device,
                                 pdeb200_write_progress progress, void* user, char* message,
                                 size_t message_len);

/* The value text of the legacy file (everything after LOOKUP_TABLE) made on
 * the host by the same formatter the GPU runs, for checking the formatter
 * without a GPU; the writers never call it. Writes at most `capacity` bytes
 * and sets *length to the full text length (PDEB200_ERR_INVALID when it did
 * not fit). out may be NULL to ask for the length. */
pdeb200_status pdeb200_vtk_values_host(const double* field, int64_t n, int32_t nx, char* out,
                                       size_t capacity, size_t* length);

#ifdef __cplusplus
}
#endif

#endif /* PDEB200_H */
