/*
 * CPU oracle: a serial C restatement of the reference bml ELLPACK / ELLBLOCK
 * thresholded-multiply path.  TEST INFRASTRUCTURE ONLY -- used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker,
 * never by the library.  Arrays use the reference layout: ELLPACK row-major
 * value[N*M], index[N*M], nnz[N]; ELLBLOCK blocks stored as separate
 * row-major bsize[ib] x bsize[jb] arrays reached through a pointer table.
 * Every function names the reference loop (file:line, relative to
 * src/C-interface/ of the bml tree) whose arithmetic and output order it
 * follows.  Compiled with -ffp-contract=off, like the reference's -std=c99
 * build, so every product and sum is separately rounded.
 */
#ifndef BML_ORACLE_H
#define BML_ORACLE_H

/* X2 = X*X thresholded; returns the largest pre-truncation row width and
 * writes trace[2] = {tr X, tr X2} (ellpack/bml_multiply_ellpack_typed.c:130-349). */
int oracle_ellpack_x2_d(int N, int M, const double *v, const int *ix, const int *nz,
                        double thr, int M2, double *v2, int *ix2, int *nz2, double *trace);
int oracle_ellpack_x2_f(int N, int M, const float *v, const int *ix, const int *nz,
                        double thr, int M2, float *v2, int *ix2, int *nz2, double *trace);
/* C = A*B thresholded, diagonal kept (ellpack/bml_multiply_ellpack_typed.c:362-553). */
int oracle_ellpack_ab_d(int N, int MA, const double *av, const int *aix, const int *anz,
                        int MB, const double *bv, const int *bix, const int *bnz,
                        double thr, int MC, double *cv, int *cix, int *cnz);
/* A = alpha*A + beta*B thresholded (ellpack/bml_add_ellpack_typed.c:50-216). */
void oracle_ellpack_add_d(int N, int MA, double *av, int *aix, int *anz, int MB,
                          const double *bv, const int *bix, const int *bnz, double alpha,
                          double beta, double thr);
/* A = A + beta*I thresholded (ellpack/bml_add_ellpack_typed.c:420-549). */
void oracle_ellpack_add_identity_d(int N, int M, double *v, int *ix, int *nz, double beta,
                                   double thr);
/* in-place threshold (ellpack/bml_threshold_ellpack_typed.c:88-133). */
void oracle_ellpack_threshold_d(int N, int M, double *v, int *ix, int *nz, double thr);
/* trace (ellpack/bml_trace_ellpack_typed.c:74-88) and trace_mult (:103-162). */
double oracle_ellpack_trace_d(int N, int M, const double *v, const int *ix, const int *nz);
double oracle_ellpack_trace_mult_d(int N, int MA, const double *av, const int *aix,
                                   const int *anz, int MB, const double *bv, const int *bix,
                                   const int *bnz);
/* B = A^T, rows in ascending source row (ellpack/bml_transpose_ellpack_typed.c:35-130,
 * serial order). */
void oracle_ellpack_transpose_d(int N, int M, const double *v, const int *ix, const int *nz,
                                double *tv, int *tix, int *tnz);
/* Gershgorin bounds {emin, emax} (ellpack/bml_normalize_ellpack_typed.c:82-175). */
void oracle_ellpack_gershgorin_d(int N, int M, const double *v, const int *ix, const int *nz,
                                 double *bounds);
/* SP2 solve with the same rules as bml_b200_sp2; returns iterations, info[6]. */
int oracle_ellpack_sp2_d(int N, int M, const double *hv, const int *hix, const int *hnz,
                         double thr, double occ, int maxiter, double tol, int stall,
                         double *dv, int *dix, int *dnz, double *info);

/* ELLBLOCK X^2 with any block sizes (ellblock/bml_multiply_ellblock_typed.c:246-442):
 * blocks[ib*MB + jp] points to block (ib, indexb[ib*MB+jp]); output blocks are
 * written to out_blocks (caller-provided storage of maxbs^2 per slot).
 * trace_quirk = 1 reproduces the reference's tr X2 stride (:410-414, which
 * steps the diagonal with bsize of the jx-list position); 0 sums the true
 * diagonal.  Returns the largest pre-truncation block-row width. */
int oracle_ellblock_x2_d(int NB, int MB, const int *bsize, double *const *blocks,
                         const int *indexb, const int *nnzb, double thr, int MB2,
                         double *const *out_blocks, int *out_indexb, int *out_nnzb,
                         double *trace, int trace_quirk);
/* The same in single precision (blocks, products and sums in float). */
int oracle_ellblock_x2_s(int NB, int MB, const int *bsize, float *const *blocks,
                         const int *indexb, const int *nnzb, double thr, int MB2,
                         float *const *out_blocks, int *out_indexb, int *out_nnzb,
                         double *trace, int trace_quirk);

#endif
