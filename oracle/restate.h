/* Test infrastructure only: plain-C restatement of the reference's solve path
 * (the oracle). Used by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline; never linked into libpdeb200.so.
 *
 * Every entry mirrors the library entry of the same name in include/pdeb200.h
 * and follows the reference CPU code cited at each function in restate.c.
 * Where the reference has no implementation (3D Krylov/MG, divergence-form k,
 * folded mixed boundaries, 3D heat) the restatement extends the cited 2D code
 * and is pinned to the reference through the special cases it does cover. */
#ifndef ORACLE_RESTATE_H
#define ORACLE_RESTATE_H

#include "pdeb200.h"
#include "pdeb200_batch.h"
#include "pdeb200_server.h"

#ifdef __cplusplus
extern "C" {
#endif

int rs_solve(const pdeb200_problem* prob, const pdeb200_options* opt, double* out,
             pdeb200_report* report);
int rs_apply(const pdeb200_problem* prob, const double* x, double* y);
int rs_residual_norms(const pdeb200_problem* prob, const double* grid, double* l2, double* linf);
int rs_time_series(const pdeb200_problem* prob, const pdeb200_time_options* topt, double* out,
                   double* frames_out);
int rs_project(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double* u,
               double* v, double* w, double* p, const pdeb200_projection_options* popt,
               pdeb200_projection_report* rep);
/* Folded system of the B200 Krylov/MG forms: b (interior rows; boundary rows 0),
 * y = A_fold x and the boundary fill of a field from its interior. */
int rs_folded_rhs(const pdeb200_problem* prob, double* b);
int rs_folded_apply(const pdeb200_problem* prob, const double* x, double* y);
int rs_fill_boundary(const pdeb200_problem* prob, double* grid);
void rs_set_threads(int n);
long rs_sizeof(int which);
void rs_set_mg_boundary_transfer(int on);

#ifdef __cplusplus
}
#endif

#endif
