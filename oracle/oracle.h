/*
 * oracle.h -- CPU restatement of the Linompss tiled SPD-solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; it exists so that tests/, the smoke check and the CPU
 * baseline leg of bench.py have an independent checker.
 *
 * Every routine restates a reference routine (citations are paths inside the
 * Linompss source tree).  The tile operations are plain triple loops with
 * 64-bit index arithmetic; the drivers issue the tile operations in exactly
 * the order the reference drivers issue their tile tasks.
 *
 * Parity pin: tests/golden/ holds outputs of the reference itself (compiled
 * from its own sources by oracle/ref.mk and linked against OpenBLAS), and
 * tests/test_oracle_golden.py checks this restatement against them.
 */
#ifndef LINOMPSS_ORACLE_H
#define LINOMPSS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Option characters follow the non-MKL ompssblas_t decoding (fpmatr.h:47-117):
 * side 'L'/'R', uplo 'L'/'U', trans 'N'/'T', diag 'N'/'U'. */

/* LAPACK dpotrf(uplo='L') on one tile (tasks_potrf.c:20-24).  Returns LAPACK
 * info: 0, or the order of the first leading minor that is not positive. */
int orc_dpotrf(int64_t n, double *A, int64_t lda);
int orc_spotrf(int64_t n, float *A, int64_t lda);

/* BLAS dtrsm (tasks_trsm.c:22-25): side/uplo/trans/diag as characters. */
void orc_dtrsm(char side, char uplo, char trans, char diag, int64_t m, int64_t n,
               double alpha, const double *A, int64_t lda, double *B, int64_t ldb);
void orc_strsm(char side, char uplo, char trans, char diag, int64_t m, int64_t n,
               float alpha, const float *A, int64_t lda, float *B, int64_t ldb);

/* BLAS dsyrk (tasks_syrk.c:19-21). */
void orc_dsyrk(char uplo, char trans, int64_t n, int64_t k, double alpha,
               const double *A, int64_t lda, double beta, double *C, int64_t ldc);
void orc_ssyrk(char uplo, char trans, int64_t n, int64_t k, float alpha,
               const float *A, int64_t lda, float beta, float *C, int64_t ldc);

/* BLAS dgemm (task_gemm.c:55-58). */
void orc_dgemm(char transa, char transb, int64_t m, int64_t n, int64_t k, double alpha,
               const double *A, int64_t lda, const double *B, int64_t ldb,
               double beta, double *C, int64_t ldc);
void orc_sgemm(char transa, char transb, int64_t m, int64_t n, int64_t k, float alpha,
               const float *A, int64_t lda, const float *B, int64_t ldb,
               float beta, float *C, int64_t ldc);

/* Tile Cholesky drivers.  Column-major: chol_rlmain.c:22-53, chol_llmain.c:23-57.
 * Hypermatrix (Ah[j*mt+i] -> b x b tile (i,j), ld=b): chol_hrlmain.c:16-37,
 * chol_hllmain.c:17-45.  Return the first non-zero tile info (the reference
 * drops it and returns 0; the product returns it, so the oracle does too). */
int orc_dchol_rl(int64_t n, int64_t b, double *A, int64_t lda);
int orc_dchol_ll(int64_t n, int64_t b, double *A, int64_t lda);
int orc_dchol_hrl(int64_t mt, int64_t b, double **Ah);
int orc_dchol_hll(int64_t mt, int64_t b, double **Ah);
int orc_schol_rl(int64_t n, int64_t b, float *A, int64_t lda);

/* Blocked left triangular solve bblas_dltrsm (bblas_trsm.h:116-202), all four
 * uplo/trans branches. */
void orc_dltrsm(char uplo, char trans, char diag, int64_t bm, int64_t m, int64_t n,
                double alpha, const double *A, int64_t lda, double *B, int64_t ldb);

/* dspdsolv_main (spdsolv_main.c:10-20): chol_rl then the two blocked solves.
 * A is m x m (ld = m), B is m x nrhs (ld = m). */
int orc_dspdsolv(int64_t m, int64_t nrhs, int64_t b, double *A, double *B);
int orc_dgetrf(int64_t m, int64_t n, int64_t b, double *A, int64_t lda, int *ipiv);
int orc_dgensolv(int64_t m, int64_t n, int64_t b, double *A, double *B);

/* Dense FP64 CG of dcg_pure (itref.c:690-925, non-preconditioned dense
 * branch, s = 1).  x holds the start vector on entry, the iterate on exit.
 * Returns -1 when ||r||/||b|| <= tol was reached, else the step count.
 * res_log (may be NULL) receives ||r_k||/||b|| for each executed step. */
int orc_dcg(int64_t n, int64_t bm, const double *A, int64_t lda, const double *b,
            double *x, double tol, int steps, double *res_log);

/* Dense iterative-refinement loop of itref.c:999-1101 (the `refit > 0`
 * branch, s = 1): x0 = CG(A, b); then up to `refit` corrections, each one a CG
 * solve of A s = r followed by the outer absolute test ||r_prev||_2 <= prec,
 * x += s and r = b - A x.  norms receives one entry per executed outer
 * iteration (entry 0 is sqrt(DBL_MAX), as in the reference, because the
 * residual of the initial solve is never dotted).  Returns the number of
 * outer iterations executed. */
int orc_ditref(int64_t n, int64_t bm, const double *A, const double *rhs, double *x,
               double prec, int refit, int it, double *norms);

/* Factor-quality and solve-quality measures used by the reference tests:
 * ||A - L L^T||_inf / (||A||_inf * n * eps) (tests/dense_tests/potrf_test.c:6-37)
 * and the normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf). */
double orc_chol_residual(int64_t n, const double *A0, int64_t lda0, const double *L, int64_t ldl);
double orc_backward_error(int64_t n, int64_t nrhs, const double *A, int64_t lda,
                          const double *X, int64_t ldx, const double *B, int64_t ldb);

/* ---- sparse refinement (itref.c, USE_SPARSE): CSR with base = vptr[0] ---- */
void orc_csrmv(int64_t n, int base, const int *vptr, const int *vpos, const double *vval, const double *x,
               double alpha, double beta, double *y);
/* block-Jacobi factors: F[k bm bm ...] = chol of diagonal block k (ld bm); 0 or 1 + failed block */
int orc_bj_setup(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval, double *F);
void orc_bj_apply(int64_t n, int64_t bm, const double *F, const double *r, double *z);
/* dcg_pure with the CSR matrix (F = NULL: no preconditioner) */
int orc_dscg(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval,
             const double *F, const double *b, double *x, double tol, int steps, double *res_log);
int orc_dsitref(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval,
                const double *F, const double *rhs, double *x, double prec, int refit, int it, double *norms);

#ifdef __cplusplus
}
#endif
#endif
