/*
 * dumses_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (C, FP64, OpenMP) of the DUMSES-Hybrid v2.2.0 Godunov MHD
 * step, used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
 * as the checker of the CUDA library.  Nothing in the product path links it.
 *
 * Every routine follows the Fortran source it names (file:line in the reference
 * project) statement by statement, in the same arithmetic order, on arrays with
 * the same bounds and column-major layout.  Build with -O2 -ffp-contract=off so
 * that no multiply-add is fused, matching a gfortran build on x86-64 without FMA.
 *
 * Pinning: the restatement is checked against the reference's only numeric
 * golden file, utils/test/fig/reference/shearing/mri/history.txt (a
 * deterministic 32x64x32 isothermal shearing-box run, 601 history rows), by
 * tests/test_oracle_golden.py.  The reference itself (Fortran) cannot be built
 * in this container: there is no Fortran compiler.
 */
#ifndef DUMSES_ORACLE_H
#define DUMSES_ORACLE_H
#include "../include/dumses_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_state or_state;

or_state *or_create(const dg_params *p);
void      or_destroy(or_state *s);

/* pointer to the state array uin(iu1:iu2,ju1:ju2,ku1:ku2,1:11), column-major */
double   *or_uin(or_state *s);
long long or_uin_size(const or_state *s);

/* the reference routines (module globals dt/time passed explicitly) */
void   or_primitive(or_state *s, double dt);          /* scheme.f90:20-91      */
double or_compute_dt(or_state *s);                    /* physics.f90:18-132    */
void   or_godunov(or_state *s, double dt, double time);/* scheme.f90:104-189   */
void   or_fargo_update(or_state *s, double dt);       /* fargo.f90:17-124      */
void   or_boundary(or_state *s, double time, double dt); /* boundary.f90:18-92 */
void   or_history_mri(or_state *s, double out[9]);    /* mri/history.f90:19-174 */
void   or_history_default(or_state *s, double out[9]); /* subroutines/history.f90:19-171, NDIM 3 */
void   or_history_1d(or_state *s, double out[3]);      /* subroutines/history.f90:37-59, NDIM 1 */
void   or_dissipation(or_state *s, double time, double dt); /* physics.f90:272-664 */

/* loop body dumses.f90:82-120; returns the dt used and advances *time */
double or_step(or_state *s, double *time);

/* Run the reference's MRI regression driver loop (dumses.f90:64-160 with the
 * history schedule of :121-126) from the current state until time > tlim,
 * writing one row per history call: time, dt, mass, maxwell, reynolds,
 * max+rey, magp, meanBx, meanBy, meanBz, divB.  Returns the number of rows
 * written (at most max_rows). */
int or_run_history(or_state *s, double tlim, double dthist, double *rows, int max_rows);

/* Intermediate arrays of the last or_godunov call, for stage-level checks.
 * which: 0 flux (if1:if2,jf1:jf2,kf1:kf2,1:8,1:ndim), 1 emfx, 2 emfy, 3 emfz
 * (iu1:iu2,...), 4 fgodunov_pre (iu1:iu2,...,1:ndim), 5 qin (iu1:iu2,...,1:8). */
double *or_array(or_state *s, int which, long long *count);

/* Initial state of one of the library's problems (DG_IC_* of dumses_gpu.h) written into
 * uin, ghosts included: the same values, bit for bit, as the library's dg_condinit, so that
 * the CPU baseline builds its workload without loading the library.  Returns DG_OK or
 * DG_ERR_ARG (unknown problem, or one that needs another ndim). */
int or_condinit(or_state *s, int ic, double beta, double amp, unsigned long long seed);

/* threads used by OpenMP loops (0 = leave the runtime default) */
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
