/*
 * lbm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the reference time step (R-IFFERY/Fortran_loadFile_mitiwing),
 * used as the checker of the CUDA path by tests/, __graft_entry__.smoke() and
 * the cpu_baseline / reference arm of bench.py. Nothing in the product links it.
 *
 * Parity unpinned: the reference ships no tests or golden vectors and cannot be
 * compiled here (Fortran + nvfortran-only cublas/cusolverDn modules, no Fortran
 * compiler in the image). The oracle is pinned by its own property tests
 * (tests/test_oracle.py) and follows the reference line by line; each function
 * cites the file:line it restates.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include "../include/lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_state ora_state;

ora_state *ora_create(const lbm_params *p);
void ora_destroy(ora_state *h);
int ora_set_boundary(ora_state *h, int wing, const double *x, const double *y, int npts);
int ora_set_motion_table(ora_state *h, const double *table, int rows, int cols);
int ora_init(ora_state *h, const double *du, const double *dv);
int ora_step(ora_state *h, double *force_row);
int ora_force_row_length(const ora_state *h);
int ora_erranalysis(ora_state *h, double *err);
void ora_get_fields(const ora_state *h, double *rho, double *u, double *v);
void ora_get_f(const ora_state *h, double *f);
void ora_set_f(ora_state *h, const double *f);
void ora_get_f0(const ora_state *h, double *f0);
void ora_get_gforce(const ora_state *h, double *gx, double *gy);
int ora_get_markers(const ora_state *h, double *xb2, double *yb2, double *solve_residual);
int ora_support_count(const ora_state *h);
int ora_step_index(const ora_state *h);
const char *ora_last_error(const ora_state *h);

/* pieces exposed for property tests */
void ora_mrt_matrices(double *matm, double *inv);          /* 81 each, row-major [row][col] */
void ora_lattice(int *e, double *w);                         /* e[9][2], w[9] */
double ora_delta(double r, int smooth);                      /* one-axis kernel value */
void ora_collide_node(const ora_state *h, const double f[9], double rho, double u, double v, double gfx,
                      double gfy, double out[9]);   /* one node of colission */
int ora_motion_row(const ora_state *h, int step_index, double *row); /* step-table row */
int ora_motion_lookup(const double *table, int rows, int cols, double t, double *row);
void ora_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
