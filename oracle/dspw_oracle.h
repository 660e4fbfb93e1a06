/*
 * dspw_oracle.h -- TEST INFRASTRUCTURE.  A plain-C FP64 restatement of the
 * reference stage path (enflo/src, enflo_scalar/src_scalar).  It is the checker
 * for the CUDA product: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it.  Nothing in the product links or calls it.
 *
 * Parity pin: each restated function follows the operation order of the
 * reference line it cites, so with the reference's compiler flags (gcc -O3,
 * no FMA contraction) it reproduces the compiled reference bit for bit; the
 * tests check that against oracle/_ref and the committed golden vectors.
 *
 * Arrays: interior cells, (nvar, Nz, Ny, Nx) planes, x fastest, FP64.
 */
#ifndef DSPW_ORACLE_H
#define DSPW_ORACLE_H
#include "../include/dspw.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_state or_state;

or_state* or_create(const dspw_desc* d);
void or_destroy(or_state* s);
void or_set_prim(or_state* s, const double* prim);
void or_get_prim(const or_state* s, double* prim);
void or_get_cons(const or_state* s, double* cons);
double or_compute_dt(or_state* s);
void or_residual(or_state* s, int rk, double* res);
/* loop body of FV::run; fixed_dt > 0 replaces the CFL step.  Returns steps taken. */
int or_step(or_state* s, int nsteps, double fixed_dt);
#define OR_DIAG_COLS 12
int or_step_diag(or_state* s, int nsteps, double fixed_dt, double* rows);
void or_time(const or_state* s, double* t, int* iter, double* dt);
/* total entropy and conserved totals (dspw_globals_out semantics) */
void or_globals(or_state* s, double* total_entropy, double* conserved5, double* ke);

/* face-level pieces */
double or_logavg(double a, double b);
void or_sp_weno(const double u[4], int corr_type, double* recl, double* recr);
void or_nn_forward(const dspw_desc* d, const double u[4], double* recl, double* recr);
/* DSP-WENO pieces exposed for the training checks: features (5), vertices (2x5). */
void or_nn_features(const double u[4], double feat[5], double vx[5], double vy[5]);
/* Euler face flux for a primitive face stencil P[ns][5] with unit normal dir,
 * cell sizes dx,dy,dz; V[ns][5] receives the entropy variables used.  ns = 4,
 * 6 for eno 3 (the reference's 2 ng_cell). */
void or_euler_face_flux(const dspw_desc* d, const double* P, int dir, double dx, double dy,
                        double dz, double* V, double flux[5]);
/* scalar face flux of a stencil u[ns] (ns as above) */
double or_scalar_face_flux(const dspw_desc* d, const double* u, int dir, double dx, double dy,
                           double dz);

#ifdef __cplusplus
}
#endif
#endif
