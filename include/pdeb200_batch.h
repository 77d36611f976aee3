/* Batched solves of many independent grids (libpdeb200).
 *
 * No counterpart in the reference: the reference solves one SolveInput per
 * call (src/backend_solve.cpp:53-211). A batch holds many problems of mixed
 * sizes and dimensions (2D and 3D, constant or divergence-form coefficients,
 * any face kinds) and solves them together on one GPU: every phase of the
 * solver is one kernel launch over a tile table that covers the matching
 * multigrid level of every member, and one refinement cycle of all phases is
 * a captured CUDA graph. Each member is solved by FP32 MG-preconditioned CG
 * (V-cycle with red-black Gauss-Seidel, FP32 or BF16 hierarchy coefficients)
 * inside FP64 iterative refinement, to a relative FP64 residual
 * |b - A u| / |b| <= tol of the boundary-folded system (the measure that
 * pdeb200_solve reports for METHOD_MG_PCG). A member's result does not depend
 * on the other members of the batch: reductions are per member in a fixed
 * order, so the same problem gives the same bits alone and in any batch made
 * with the same options.
 *
 * Tile shapes and smoother schedule come from pdeb200_batch_options or from
 * the autotuner, which times candidate schedules on the batch itself and
 * keeps the winner in an on-disk cache keyed by the device and the batch's
 * shapes. As members converge, the tile tables are rebuilt for the
 * unfinished ones (compaction), which changes no member's numbers. */
#ifndef PDEB200_BATCH_H
#define PDEB200_BATCH_H

#include "pdeb200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdeb200_batch pdeb200_batch;

typedef struct {
  int32_t device;
  int32_t tile_x;          /* 2D tile width in nodes (32 or 64); 0 = default 32 */
  int32_t tile_y;          /* 2D tile height in nodes (8, 16 or 32); 0 = default 16 */
  int32_t tile_z;          /* 3D tile depth in planes (32 x 8 columns); 0 = default 8 */
  int32_t pre_smooth;      /* red-black sweeps before/after the coarse correction; 0 = 2 */
  int32_t post_smooth;
  int32_t coarse_sweeps;   /* FP64 sweeps on each member's coarsest level; 0 = 16 */
  int32_t max_inner;       /* inner FP32 MG-PCG iterations per refinement step; 0 = 40 */
  int32_t max_outer;       /* FP64 residual evaluations; 0 = 12 */
  int32_t bf16_coefficients; /* 1: hierarchy k stored as BF16 */
  int32_t no_graph;        /* 1: launch the cycle's kernels directly instead of a graph */
  int32_t autotune;        /* 1: time candidate schedules at create and keep the fastest */
  double inner_tol;        /* inner relative tolerance; 0 = 1e-4. A member's last refinement step
                              stops once the reduction left to the target is reached */
  const char* tune_cache;  /* autotuner cache file; NULL = $PDEB200_TUNE_CACHE, else none */
  void* stream;            /* cudaStream_t for all work; NULL = the batch's own stream */
  int32_t no_compact;      /* 1: keep every member's tiles in the launches until the solve ends */
  int32_t reserved[7];
} pdeb200_batch_options;

typedef struct {
  int32_t members;
  int32_t converged;       /* members with status OK */
  int32_t cycles;          /* refinement cycles launched (graph replays) */
  int32_t max_levels;      /* deepest member hierarchy */
  int64_t kernel_launches;
  int64_t tiles_level0;
  int64_t nodes;           /* total level-0 nodes */
  int64_t device_bytes;    /* device memory held by the batch */
  double device_ms;        /* last solve, device time */
  double tune_ms;          /* autotuning time at create (0 when cached or off) */
  int32_t tuned_from_cache;
  int32_t graph;           /* 1 when the cycle ran as a CUDA graph */
  int32_t compactions;     /* times the tables were rebuilt for the unfinished members */
  int32_t reserved[5];
} pdeb200_batch_stats;

void pdeb200_batch_default_options(pdeb200_batch_options* opt);

/* Builds a batch: validates and uploads every member (coefficients, faces,
 * right-hand side f when given), builds each member's hierarchy and the tile
 * tables, and (autotune) picks the schedule. Members must have COEF_CONST or
 * COEF_DIVK and at least one side of 5 or more nodes. The problems' arrays
 * are read during the call only. On failure *out is NULL and `message` (may
 * be NULL) receives the reason. */
pdeb200_status pdeb200_batch_create(const pdeb200_problem* members, int32_t count,
                                    const pdeb200_batch_options* opt, pdeb200_batch** out,
                                    char* message, size_t message_len);

/* Total level-0 nodes and the offset of `member` in the packed arrays below
 * (members in order, each nx*ny*nz values in the reference's layout). */
int64_t pdeb200_batch_nodes(const pdeb200_batch* b);
int64_t pdeb200_batch_offset(const pdeb200_batch* b, int32_t member);

/* Replaces every member's right-hand side f (packed; host or device memory). */
pdeb200_status pdeb200_batch_load_rhs(pdeb200_batch* b, const double* f_packed, int32_t mem_space);

/* Solves every member to |b - A u| / |b| <= tol. reports: NULL or `count`
 * entries (iterations = inner iterations, outer_iterations = FP64
 * refinement steps, rel_residual = final FP64 relative residual). Returns OK
 * when every member converged, else the first failing member's status. */
pdeb200_status pdeb200_batch_solve(pdeb200_batch* b, double tol, pdeb200_report* reports,
                                   pdeb200_batch_stats* stats);

/* Copies every member's solution (boundary nodes included) into `out_packed`. */
pdeb200_status pdeb200_batch_read(pdeb200_batch* b, double* out_packed, int32_t mem_space);

/* Copies one member's solution (nx*ny*nz values) into `out` (host or device). */
pdeb200_status pdeb200_batch_read_member(pdeb200_batch* b, int32_t member, double* out, int32_t mem_space);

/* Options in effect (after defaults and autotuning). */
pdeb200_status pdeb200_batch_get_options(const pdeb200_batch* b, pdeb200_batch_options* opt);

void pdeb200_batch_destroy(pdeb200_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* PDEB200_BATCH_H */
