/* Serving: a device-resident request loop over libpdeb200 (one GPU).
 *
 * No counterpart in the reference, which solves one SolveInput per process
 * call (src/main.cpp, src/backend_solve.cpp:53-211). A server takes Poisson /
 * diffusion solves, explicit heat runs and pressure projections as they
 * arrive, admits each one when its device memory fits the HBM budget, and
 * runs admitted work concurrently on several lanes (one CUDA stream, solver
 * context and host thread each), so requests that arrive while others are on
 * the GPU overlap with them.
 *
 * Poisson requests in MIXED precision are continuously batched: when a lane
 * is free it takes every admitted Poisson request waiting (up to max_batch)
 * and solves them as one pdeb200_batch (FP32 MG-PCG inside FP64 refinement,
 * one launch per phase for the whole group). In FP64 precision each Poisson
 * request runs the plain FP64 MG-PCG path (pdeb200_solve). Heat runs use the
 * forward-Euler series of pdeb200_time_series; projections use
 * pdeb200_project_velocity's algorithm. A request's result does not depend on
 * what else is in flight: with fixed batch options (and single_below off) the
 * same request gives the same bits alone and in any mix. */
#ifndef PDEB200_SERVER_H
#define PDEB200_SERVER_H

#include "pdeb200.h"
#include "pdeb200_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdeb200_server pdeb200_server;

typedef enum {
  PDEB200_REQ_POISSON = 0,     /* steady solve of the problem to tol (relative, folded system) */
  PDEB200_REQ_HEAT = 1,        /* `steps` forward-Euler steps of u_t-form problem from u0 */
  PDEB200_REQ_PROJECTION = 2   /* one Chorin projection of (u, v[, w]) with pressure p */
} pdeb200_request_kind;

typedef struct {
  int32_t device;
  int32_t lanes;             /* concurrent lanes (streams); 0 = 4 */
  int32_t max_batch;         /* Poisson requests per batched group; 0 = 64 (groups on several lanes
                                overlap one group's last, sparse cycles with another's full ones) */
  int32_t precision;         /* PDEB200_MIXED (batched groups) or PDEB200_FP64 (plain MG-PCG path) */
  int64_t hbm_budget_bytes;  /* admission budget; 0 = 80% of the device's free memory at create */
  int32_t queue_capacity;    /* queued (not yet admitted) requests; 0 = 65536 */
  int32_t single_below;      /* MIXED: while fewer than this many Poisson requests wait, a free lane
                                takes one and solves it on its own grid (FP32 MG-PCG inside FP64
                                refinement, pdeb200_solve with precision MIXED) instead of as a
                                batched group, so light load pays no batching latency; results then
                                agree with a batched solve to the tolerance, not bitwise.
                                0 or 1 = always batch */
  pdeb200_batch_options batch; /* options of the batched groups (autotune is ignored) */
  int32_t reserved[8];
} pdeb200_server_options;

typedef struct {
  int32_t kind;              /* pdeb200_request_kind */
  int32_t steps;             /* HEAT: forward-Euler steps */
  /* POISSON, HEAT. Host arrays (mem_space HOST) are copied at submit; device
   * arrays (mem_space DEVICE) are used in place and must stay valid until the
   * request completes, and `out` is then a device pointer. */
  const pdeb200_problem* problem;
  double tol;                /* POISSON: relative residual; 0 = 1e-10 */
  double t_start, dt;        /* HEAT */
  /* PROJECTION (host arrays, copied at submit; nz <= 1 is 2D) */
  int32_t nx, ny, nz, max_iter;
  double dx, dy, dz, proj_dt, proj_tol;
  const double *u, *v, *w, *p;
  /* Result: host buffer the server fills before the request completes.
   * POISSON/HEAT: nx*ny*nz values; PROJECTION: u, v, (w,) p packed. */
  double* out;
} pdeb200_request;

typedef struct {
  int64_t id;
  int32_t status;            /* pdeb200_status of the request */
  int32_t kind;
  double queue_ms;           /* submit -> admitted to a lane */
  double run_ms;             /* admitted -> result written */
  double latency_ms;         /* submit -> result written */
  int32_t iterations;        /* inner (batched) / MG-PCG / CG iterations */
  int32_t group_size;        /* requests solved together with this one */
  double rel_residual;
  char message[128];
} pdeb200_result;

typedef struct {
  int64_t submitted, completed, failed, rejected;
  int64_t in_flight, queued;
  int64_t bytes_in_use, bytes_peak, budget_bytes;
  int32_t lanes_busy_peak;   /* most lanes running at once */
  int32_t reserved0;
  double p50_ms, p99_ms, max_ms;   /* latency over completed requests since the last reset */
  double elapsed_s;                /* since the last reset */
  double solves_per_s;             /* completed / elapsed_s */
  int32_t reserved[8];
} pdeb200_server_stats;

pdeb200_status pdeb200_server_create(const pdeb200_server_options* opt, pdeb200_server** out, char* message,
                                     size_t message_len);
/* Queues a request (inputs are copied; `out` must stay valid until the
 * request completes). PDEB200_ERR_BUSY when the queue is full,
 * PDEB200_ERR_OOM when the request alone exceeds the HBM budget. */
pdeb200_status pdeb200_server_submit(pdeb200_server* s, const pdeb200_request* req, int64_t* id);
/* Waits up to timeout_ms (< 0: forever) for request `id`; PDEB200_ERR_TIMEOUT
 * if it is still running. A completed request's record is released by the
 * first successful wait. */
pdeb200_status pdeb200_server_wait(pdeb200_server* s, int64_t id, double timeout_ms, pdeb200_result* res);
/* Waits until nothing is queued or running (timeout as above). */
pdeb200_status pdeb200_server_drain(pdeb200_server* s, double timeout_ms);
pdeb200_status pdeb200_server_get_stats(pdeb200_server* s, pdeb200_server_stats* st, int32_t reset);
void pdeb200_server_destroy(pdeb200_server* s);

#ifdef __cplusplus
}
#endif

#endif /* PDEB200_SERVER_H */
