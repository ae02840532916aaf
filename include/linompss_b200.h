/*
 * linompss_b200.h -- C ABI of the B200 (sm_100a) tiled SPD-solve library.
 *
 * Drop-in for the Linompss tiled SPD-solve path.  The first group of entry
 * points keeps the reference's names, argument order and storage
 * conventions (column-major, leading dimension lda, tile size b, and the
 * hypermatrix tile table Ah[j*mt+i] -> b x b tile (i,j) with ld = b); each
 * one cites the reference declaration it replaces.  They take HOST pointers,
 * copy to the GPU, compute there and copy back, and are synchronous like the
 * reference after `#pragma omp taskwait`.
 *
 * Return codes (a documented superset of the reference, which always
 * returns 0):
 *     0   success
 *    >0   LAPACK-style: the order of the first leading minor that is not
 *         positive definite (the factorization stopped there)
 *    <0   an LNB_E* error (argument, device, or scheduler timeout);
 *         lnb_last_error() gives a message.
 *
 * The lnb_* entry points are B200-specific additions: device-pointer forms
 * that run on a caller stream (cudaStream_t passed as void*), the
 * mixed-precision solver with FP64 iterative refinement, and the batched
 * solver.  All device pointers must be CUDA device memory of the current
 * device.
 *
 * Host code of this library is C; kernels are CUDA for sm_100a only.  There
 * is no CPU fallback: without a usable B200 every entry point returns
 * LNB_ENODEV.
 */
#ifndef LINOMPSS_B200_H
#define LINOMPSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LNB_EXPORT __attribute__((visibility("default")))

/* ---- error codes -------------------------------------------------------- */
#define LNB_OK          0
#define LNB_EINVAL    (-1)   /* bad argument (size, leading dimension, option) */
#define LNB_ENODEV    (-2)   /* no usable sm_100 device */
#define LNB_ECUDA     (-3)   /* CUDA runtime error */
#define LNB_ENOMEM    (-4)   /* device allocation failed */
#define LNB_ETIMEOUT  (-5)   /* a device-side dependency wait ran out */
#define LNB_ENOCONV   (-6)   /* refinement did not reach the requested accuracy */
#define LNB_ETOOBIG   (-7)   /* size beyond a fixed capacity of the entry point */

/* ---- BLAS option descriptor ---------------------------------------------
 * ompssblas_t / ompsslapack_t (fpmatr.h:14-35).  This library decodes the
 * non-MKL form: .s points at a string whose first character is the option
 * ('L'/'R' side, 'L'/'U' uplo, 'N'/'T' trans, 'N'/'U' diag), exactly as
 * TEST_LEFT/TEST_LOWER/... do (fpmatr.h:47-117). */
typedef union { int e; char *s; } ompssblas_t;
typedef union { char e; char *s; } ompsslapack_t;

/* ======================================================================== */
/* 1. Reference entry points (host pointers, synchronous)                    */
/* ======================================================================== */

/* Column-major tile Cholesky, A = L L^T, lower triangle overwritten by L,
 * upper triangle untouched.  `t` (sub-tile size) is accepted and unused, as
 * in the reference.  Replace ompss_dense_chol.h:40-46 / ompss_dense_chol.c:26-41
 * (right-looking dchol_rl chol_rlmain.c:22-53, left-looking dchol_ll
 * chol_llmain.c:23-57).  Both variants produce the same factor; on the GPU
 * they run the same right-looking device schedule. */
LNB_EXPORT int ompss_dchol_rl(int n, int b, int t, double *A, int lda);
LNB_EXPORT int ompss_dchol_ll(int n, int b, int t, double *A, int lda);
LNB_EXPORT int ompss_schol_rl(int n, int b, int t, float *A, int lda);
LNB_EXPORT int ompss_schol_ll(int n, int b, int t, float *A, int lda);

/* Hypermatrix tile Cholesky: Ah[j*mt+i] points at tile (i,j), b x b,
 * column-major with ld = b (chol_hsetup.c:29-34); only tiles with i >= j are
 * read or written.  The first argument is the tile count mt (the header
 * calls it n; ompss_dense_chol.c:20 passes it as mt).  Replace
 * ompss_dense_chol.h:15-33 (dchol_hrl chol_hrlmain.c:16-37, dchol_hll
 * chol_hllmain.c:17-45) and the nested forms ompss_dense_chol.h:49-55
 * (dchol_nrl/nll, whose extra sub-tile level is internal blocking). */
LNB_EXPORT int ompss_dchol_hrl(int mt, int b, int t, double **Ah);
LNB_EXPORT int ompss_dchol_hll(int mt, int b, int t, double **Ah);
LNB_EXPORT int ompss_dchol_nhrl(int mt, int b, int t, double **Ah);
LNB_EXPORT int ompss_dchol_nhll(int mt, int b, int t, double **Ah);
LNB_EXPORT int ompss_schol_hrl(int mt, int b, int t, float **Ah);
LNB_EXPORT int ompss_schol_hll(int mt, int b, int t, float **Ah);

/* SPD solve A X = B: Cholesky, then forward L Y = B and backward L^T X = Y.
 * A is m x m (ld = m) and is overwritten by L; B is m x nrhs (ld = m) and is
 * overwritten by X.  Replaces spdsolv_main.h:20 / spdsolv_main.c:10-20. */
LNB_EXPORT int dspdsolv_main(int m, int nrhs, int b, double *A, double *B);
LNB_EXPORT int sspdsolv_main(int m, int nrhs, int b, float *A, float *B);

/* Blocked left triangular solve op(A) X = alpha B, B overwritten by X.
 * Replaces trsm/ompss_trsm.h:20-24 (-> BBLAS_LTRSM bblas_trsm.h:116-202).
 * The reference implements side = left only (trsm_main.c:9-14); so does
 * this library (side = 'R' returns LNB_EINVAL instead of printing). */
LNB_EXPORT int ompss_dtrsm(ompssblas_t side, ompssblas_t uplo, ompssblas_t trans,
                           ompssblas_t diag, int m, int n, int b, double alpha,
                           double *A, int lda, double *B, int ldb);

/* Blocked symmetric rank-k update on the triangle `uplo` of C:
 * C = alpha op(A) op(A)^T + beta C, op(A) = A (n x k) for trans 'N', A^T
 * (A k x n) for 'T'; the other triangle is not touched.  Replaces
 * syrk/ompss_syrk.h:20,22 (-> SYRK_MAIN syrk_main.c, tile GEMM/SYRK tasks of
 * width b).  b is the reference's tile size; the GPU computes the triangle in
 * one launch, so b only has to be positive.  The reference's first k-chunk is
 * always b wide (syrk_main.c), so for k < b it reads past column k; this
 * library follows BLAS for every k.  ompss_ssyrk computes in FP64 and rounds
 * the result once.  Returns 0 or LNB_E* (the reference returns void). */
LNB_EXPORT int ompss_dsyrk(ompssblas_t uplo, ompssblas_t trans, int b, int n, int k, double alpha,
                           double *A, int lda, double beta, double *C, int ldc);
LNB_EXPORT int ompss_ssyrk(ompssblas_t uplo, ompssblas_t trans, int b, int n, int k, float alpha,
                           float *A, int lda, float beta, float *C, int ldc);

/* Tile-task ABI: one BLAS/LAPACK operation on one tile, run on the GPU.
 * Replace tasks_potrf.h:24-28, tasks_trsm.h:23-27, tasks_syrk.h:20-24,
 * task_gemm.h:27-31 (exported from libbblas with the trailing OmpSs priority
 * `p`, accepted and unused).  task_dpotrf returns LAPACK info, which the
 * reference discards (tasks_potrf.c:22-23); the others return 0 or LNB_E*. */
LNB_EXPORT int task_dpotrf(ompsslapack_t uplo, int n, double *A, int lda, int p);
LNB_EXPORT int task_dtrsm(ompssblas_t side, ompssblas_t uplo, ompssblas_t trans,
                          ompssblas_t diag, int bm, int bn, double alpha, double *A,
                          int lda, double *B, int ldb, int p);
LNB_EXPORT int task_dsyrk(ompssblas_t uplo, ompssblas_t trans, int n, int k, double alpha,
                          double *A, int lda, double beta, double *C, int ldc, int p);
LNB_EXPORT int task_dgemm(ompssblas_t transa, ompssblas_t transb, int bm, int bn, int bk,
                          double alpha, double *A, int lda, double *B, int ldb, double beta,
                          double *C, int ldc, int p);

/* Dense FP64 solver of dcg_pure (itref.c:690-925), non-preconditioned dense
 * branch with s = 1: x (length n) is the start vector on entry and the
 * iterate on exit; stops at ||r||_2/||b||_2 <= tol or after `steps` steps.
 * Returns -1 if converged, else the number of steps (the reference's own
 * convention, itref.c:922-924).  The recurrence is the reference's as it
 * executes: its direction update runs with the old and new residual ratio
 * fixed at 1 and with aliased operands, so it computes p = 2 r, a damped
 * steepest descent rather than textbook CG.  bm is the reference's
 * row-block size and only affects the order of partial sums there. */
LNB_EXPORT int ompss_dcg(int n, int bm, const double *A, int lda, const double *b, double *x,
                         double tol, int steps);

/* Dense iterative refinement of itref.c:999-1101 (refit > 0 branch, s = 1):
 * x0 = dcg(A, b); then up to `refit` corrections s = dcg(A, r), stopping when
 * the previous residual's 2-norm is <= prec (absolute), else x += s,
 * r = b - A x.  The reference keeps this loop inside main(); this entry point
 * uses its argument conventions.  norms (may be NULL, length refit) receives
 * the per-iteration residual norms of itref_norms.log.  Returns the number of
 * outer iterations executed (> 0) or LNB_E*. */
LNB_EXPORT int ompss_ditref(int n, int bm, const double *A, int lda, const double *b,
                            double *x, double prec, int refit, int it, double *norms);

/* Sparse refinement: itref.c built with USE_SPARSE (the refinement loop of
 * itref.c:999-1101 and dcg_pure itref.c:690-925 over a sparse matrix).  A is
 * n x n, symmetric positive definite, in CSR with both triangles stored (the
 * reference's hbmat_t after dhb_sym_expand, hb.h:27-59): row pointers
 * vptr[n+1], column indices vpos, values vval, zero- or one-based (the base
 * is vptr[0], as the reference's one2zero reads it).  is_precond != 0: the
 * inner solver uses the reference's block-Jacobi preconditioner
 * (itref_setup.c:55-93): Cholesky, natural ordering, of every complete
 * bm x bm diagonal block, applied as z = L^-T L^-1 r (bsblas_dcholsolv2,
 * bsblas_csrmm.h:498); bm <= 512 here.  The recurrence is the reference's as
 * it executes (see ompss_dcg): alpha1 = <r, z>, direction update p = 2 z,
 * stop at sqrt(alpha1)/||b||_2 <= tol.  ompss_dscg: x is the start vector on
 * entry and the iterate on exit; returns -1 if converged, else the steps.
 * ompss_dsitref: arguments and return as ompss_ditref.  A diagonal block that
 * is not positive definite returns LNB_EINVAL naming the block. */
LNB_EXPORT int ompss_dscg(int n, int bm, const int *vptr, const int *vpos, const double *vval,
                          const double *b, double *x, double tol, int steps, int is_precond);
LNB_EXPORT int ompss_dsitref(int n, int bm, const int *vptr, const int *vpos, const double *vval,
                             const double *b, double *x, double prec, int refit, int it,
                             int is_precond, double *norms);
/* MatrixMarket coordinate file ("real" or "integer", "general" or
 * "symmetric") to zero-based CSR with ascending columns in every row; a
 * symmetric file's off-diagonal entries appear in both triangles (the input
 * the sparse refinement wants; the reference reads Harwell-Boeing files with
 * readHB_newmat_double, itref_config.c:228-241).  The arrays are allocated
 * here; release them with lnb_mm_free.  Returns 0 or LNB_E*. */
LNB_EXPORT int lnb_mm_read_csr(const char *path, int *n, int **vptr, int **vpos, double **vval);
LNB_EXPORT void lnb_mm_free(int *vptr, int *vpos, double *vval);

/* ======================================================================== */
/* 2. Device-pointer entry points (run on `stream`, asynchronous)            */
/* ======================================================================== */
/* dA: n x n FP64, column-major, ld = lda, device memory.  *info_dev (device
 * int, may be NULL) receives the LAPACK-style info.  Returns LNB_E* for
 * argument/launch errors; the factorization itself completes on the
 * stream. */
LNB_EXPORT int lnb_dchol_dev(int n, int b, double *dA, int lda, int *info_dev, void *stream);
LNB_EXPORT int lnb_schol_dev(int n, int b, float *dA, int lda, int *info_dev, void *stream);

/* FP64 tile Cholesky that allocates no device memory.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc: code whose device
 * memory is owned by another manager (a caching allocator or a fixed arena
 * holding the whole HBM), and code on a latency-critical path where
 * cudaMalloc's implicit synchronization is not acceptable.
 * Same result as lnb_dchol_dev (A = L L^T in place, lower), computed on the
 * caller's stream only.  Its scratch (block inverses + status word) is a
 * fixed file-scope device array of 256 KB held by every GPU that loads the
 * library until exit; tile sizes b > 1024 are rejected with LNB_ETOOBIG.
 * The first call on a device looks up that array's device address and
 * keeps it; make that first call before any stream capture.  Under lazy
 * module loading that first call may also load the library's kernels, which
 * the CUDA driver does with its own memory.  cudaDeviceReset destroys the
 * array with the context, so do not call this entry point again after a
 * reset in the same process.  All calls share the array: calls that overlap
 * on the GPU (other streams, other host threads) race. */
LNB_EXPORT int lnb_dchol_noalloc_dev(int n, int b, double *dA, int lda, int *info_dev, void *stream);

/* Schedule of the FP64 factorizations (ompss_dchol_*, dspdsolv_main,
 * lnb_dchol_dev, lnb_dposv_dev).  Process-wide setting; the environment
 * variable LNB_CHOL_SCHED ("dag" / "streams") overrides it.
 *   LNB_SCHED_STREAMS: right-looking steps issued by the host on two streams
 *     (diagonal factor and panel solve on a high-priority stream, the big
 *     fused DMMA trailing updates behind them): best for large n.
 *   LNB_SCHED_DAG: one persistent launch that walks the tile task DAG on the
 *     device (64 x 64 tiles handed out by an atomic ticket in priority order,
 *     dependencies tracked by per-tile flags, every wait bounded): best where
 *     the critical path dominates.  The tile size b only shapes the stream
 *     schedule; the DAG uses its own 64-wide tiles (the factor is the same up
 *     to rounding).
 *   LNB_SCHED_AUTO (default): the device DAG for n <= 4096, streams above. */
#define LNB_SCHED_AUTO     0
#define LNB_SCHED_STREAMS  1
#define LNB_SCHED_DAG      2
LNB_EXPORT void lnb_set_chol_schedule(int sched);

/* Triangular solves with the lower factor: trans 'N' solves L Y = B,
 * 'T' solves L^T X = B, 'B' (both) solves L L^T X = B.  dB: n x nrhs, ld = ldb. */
LNB_EXPORT int lnb_dpotrs_dev(int n, int nrhs, const double *dL, int lda, double *dB, int ldb,
                              char which, void *stream);
LNB_EXPORT int lnb_spotrs_dev(int n, int nrhs, const float *dL, int lda, float *dB, int ldb,
                              char which, void *stream);

/* Factor + solve: dA overwritten by L, dB by X. */
LNB_EXPORT int lnb_dposv_dev(int n, int nrhs, int b, double *dA, int lda, double *dB, int ldb,
                             int *info_dev, void *stream);

/* Generic blocked triangular solve on device memory, ompss_dtrsm semantics
 * (left side; uplo/trans/diag as characters). */
LNB_EXPORT int lnb_dtrsm_dev(char uplo, char trans, char diag, int m, int n, double alpha,
                             const double *dA, int lda, double *dB, int ldb, void *stream);

/* Device forms of the tile BLAS-3 tasks on the FP64 tensor cores (DMMA):
 * C = alpha op(A) op(B) + beta C (task_dgemm, task_gemm.c:55-58) and
 * C = alpha op(A) op(A)^T + beta C on triangle uplo of C (task_dsyrk,
 * tasks_syrk.c:19-21).  Options as characters ('N'/'T', 'L'/'U'); beta == 0
 * does not read C.  Asynchronous on `stream`. */
LNB_EXPORT int lnb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double *dA,
                             int lda, const double *dB, int ldb, double beta, double *dC, int ldc, void *stream);
LNB_EXPORT int lnb_dsyrk_dev(char uplo, char trans, int n, int k, double alpha, const double *dA, int lda,
                             double beta, double *dC, int ldc, void *stream);

/* The refinement's matrix product Y = A X for symmetric A given by its lower
 * triangle (the strict upper part of dA is not read), FP64.  Replaces the
 * reference's bblas_dgemm matvec over the full stored A (itref.c:1086,1094),
 * which reads both triangles.  dX, dY: n x nrhs with ld = n; the columns of Y
 * are sums in an unspecified order (atomic accumulation). */
LNB_EXPORT int lnb_dsymv_dev(int n, int nrhs, const double *dA, int lda, const double *dX, double *dY,
                             void *stream);

/* ---- tile LU with partial pivoting and the general solve ----------------- */
/* ompss_dgetrf (ompss_lu.h:19, dlu_main lu_main.c:5-27): P A = L U in place,
 * A m x n column-major (ld lda), b the panel width of the pivot convention.
 * IPIV (min(m, n) ints) receives the reference's convention: for the b-wide
 * panel starting at row j, IPIV[j + k] is the pivot row of column j + k,
 * 1-based and relative to row j (LAPACK dgetrf's output for the panel).
 * Returns 0, or the 1-based column of the first exactly zero pivot (LAPACK
 * info; the factorization completes); < 0 on error.  The reference's
 * functions return void.  The _ll drivers (ompss_lu.h:23-25) give the same
 * factorization.  s*: FP32 arrays, computed in FP64 on the device. */
LNB_EXPORT int ompss_dgetrf(int m, int n, int b, double *A, int lda, int *IPIV);
LNB_EXPORT int ompss_sgetrf(int m, int n, int b, float *A, int lda, int *IPIV);
LNB_EXPORT int ompss_dgetrf_ll(int m, int n, int b, double *A, int lda, int *IPIV);
LNB_EXPORT int ompss_sgetrf_ll(int m, int n, int b, float *A, int lda, int *IPIV);
/* dgensolv_main (gensolv_main.h, gensolv_main.c:10-25): A (m x m, ld m) -> its
 * LU factors, B (m x n, ld m) -> A^-1 B. */
LNB_EXPORT int dgensolv_main(int m, int n, int b, double *A, double *B);
LNB_EXPORT int sgensolv_main(int m, int n, int b, float *A, float *B);
/* device forms: dipiv receives LAPACK pivots (1-based, global rows);
 * info_dev (may be NULL) the info value; asynchronous on `stream`.  Every LU
 * entry point takes at most 32768 rows (LNB_ETOOBIG beyond). */
LNB_EXPORT int lnb_dgetrf_dev(int m, int n, double *dA, int lda, int *dipiv, int *info_dev, void *stream);
LNB_EXPORT int lnb_dgetrs_dev(int n, int nrhs, const double *dLU, int lda, const int *dipiv, double *dB, int ldb,
                              void *stream);

/* ======================================================================== */
/* 3. Mixed precision: low-precision factor + FP64 iterative refinement       */
/* ======================================================================== */
#define LNB_FACTOR_FP64    0   /* plain FP64 (DMMA updates) */
#define LNB_FACTOR_FP32    1   /* FP32 storage, SIMT FP32 updates */
#define LNB_FACTOR_TF32X3  2   /* FP32 storage, 3xTF32 split on tcgen05 */
#define LNB_FACTOR_BF16    3   /* per-tile-scaled BF16 on tcgen05, FP32 accumulate */
#define LNB_FACTOR_TF32    4   /* FP32 storage, one TF32 product on tcgen05 */

/* Update path of the FP32 factorizations (ompss_schol_*, lnb_schol_dev):
 * LNB_FACTOR_FP32, LNB_FACTOR_TF32X3 (default), LNB_FACTOR_TF32 or
 * LNB_FACTOR_BF16.  Process-wide setting. */
LNB_EXPORT void lnb_set_factor_mode(int mode);

typedef struct {
    int    factor;          /* LNB_FACTOR_* */
    int    max_iter;        /* outer refinement iterations (default 30) */
    double tol;             /* stop at normwise backward error <= tol; 0 -> 10*n*eps */
    int    equilibrate;     /* symmetric diagonal scaling before the factor */
    int    allow_pcg;       /* fall back to CG preconditioned by the factor */
    int    pcg_max_iter;    /* default 200 */
} lnb_ir_opts;

typedef struct {
    int    iterations;      /* outer refinement iterations executed */
    int    pcg_iterations;  /* PCG steps if the fallback ran, else 0 */
    int    used_pcg;        /* 1 if the PCG fallback ran */
    int    refactored_tiles;/* diagonal tiles refactored in FP64 */
    double backward_error;  /* ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf), max over rhs */
    double factor_ms;       /* device time of the factorization */
    double solve_ms;        /* device time of solves + refinement */
    int    info;            /* factorization info after fallbacks */
} lnb_ir_result;

LNB_EXPORT void lnb_ir_default_opts(lnb_ir_opts *opts);

/* Solve A X = B to FP64 backward error with a low-precision factor.
 * A (n x n FP64, ld lda) is NOT modified; B (n x nrhs) is read, X written.
 * Device-pointer form: */
LNB_EXPORT int lnb_dsposv_ir_dev(int n, int nrhs, int b, const double *dA, int lda,
                                 const double *dB, int ldb, double *dX, int ldx,
                                 const lnb_ir_opts *opts, lnb_ir_result *res, void *stream);
/* Host-pointer form (copies in and out): */
LNB_EXPORT int lnb_dsposv_ir(int n, int nrhs, int b, const double *A, int lda, const double *B,
                             int ldb, double *X, int ldx, const lnb_ir_opts *opts,
                             lnb_ir_result *res);

/* ======================================================================== */
/* 4. Batched uneven SPD solves                                               */
/* ======================================================================== */
/* count independent systems; system s has order n[s] <= 512 and nrhs[s] <= 8.
 * A_s at dA + a_off[s] (n x n, ld n), B_s/X_s at dB + b_off[s] (n x nrhs,
 * ld n).  A is not modified; X_s written at dX + b_off[s].  mode
 * LNB_FACTOR_FP32 factors in FP32 and refines in FP64; LNB_FACTOR_FP64 is
 * the plain FP64 factor+solve.  info_dev[s] (may be NULL) gets each system's
 * info; iters_dev[s] (may be NULL) the refinement iterations. */
LNB_EXPORT int lnb_batched_posv_dev(int count, const int *n_dev, const int *nrhs_dev,
                                    const int64_t *a_off_dev, const int64_t *b_off_dev,
                                    const double *dA, const double *dB, double *dX,
                                    int mode, int max_iter, int *info_dev, int *iters_dev,
                                    void *stream);
/* Autotuner: times the candidate launch shapes of the persistent solver on
 * this batch (synchronous): CTA size (256 / 512 threads), systems resident per
 * SM (1 / 2) and processing order (largest first / largest and smallest
 * interleaved), and keeps the fastest for later lnb_batched_posv_dev calls of
 * the same mode.  Returns the chosen CTA size; lnb_batched_config reports the
 * whole shape.  Each system's A_s is n x n FP64 with both triangles stored. */
LNB_EXPORT int lnb_batched_autotune(int count, const int *n_dev, const int *nrhs_dev,
                                    const int64_t *a_off_dev, const int64_t *b_off_dev,
                                    const double *dA, const double *dB, double *dX,
                                    int mode, int max_iter, void *stream);
LNB_EXPORT int lnb_batched_config(int mode, int *cta_threads, int *ctas_per_sm, int *interleave);
/* Multi-GPU split of one batch (host only, no device work): the systems in
 * decreasing order of estimated cost n^3/3 + 2 n^2 nrhs (equal costs: lower
 * index first), each given to the part with the least cost so far (ties: lower
 * part) -- longest-processing-time first.  owner[s] receives the part (0 ..
 * parts-1) of system s; load[p] (may be NULL) the estimated flops of part p.
 * The result depends only on the arguments, so every rank computes the same
 * split.  Returns 0 or LNB_EINVAL.  (The reference has no batched solver.) */
LNB_EXPORT int lnb_batched_partition(int count, const int *n, const int *nrhs, int parts, int *owner,
                                     double *load);

/* ======================================================================== */
/* 5. Runtime                                                                 */
/* ======================================================================== */
LNB_EXPORT const char *lnb_last_error(void);
LNB_EXPORT const char *lnb_version(void);
/* Release the cached device workspace of the calling thread's device. */
LNB_EXPORT void lnb_release_workspace(void);
/* Bound (in microseconds of device time) on every device-side dependency
 * wait; a wait that runs out makes the call return LNB_ETIMEOUT.  Default
 * 2,000,000 (2 s). */
LNB_EXPORT void lnb_set_wait_limit_us(long long us);

/* ---- diagnostics ---------------------------------------------------------
 * Launch counting and live timing of the trailing-update kernels (the
 * dominant kernel of the factorization).  When enabled, each update launch
 * is bracketed by CUDA events on the stream it runs on; lnb_prof_read
 * synchronizes those events and returns totals since the last reset. */
typedef struct {
    long long launches;        /* kernels launched by this library */
    long long update_launches; /* trailing-update launches timed */
    double    update_ms;       /* their summed device time */
    double    update_flops;    /* their algorithmic flops (2 per multiply-add) */
    double    update_bytes;    /* their algorithmic operand bytes (read P twice, C read+write) */
} lnb_prof_t;
LNB_EXPORT void lnb_prof_enable(int on);
LNB_EXPORT void lnb_prof_reset(void);
LNB_EXPORT int  lnb_prof_read(lnb_prof_t *out);

/* Self-test of the bounded device-side waits: launches a solve DAG in which
 * one dependency is never satisfied and returns what the call reports
 * (LNB_ETIMEOUT when the bound works).  wait_us bounds the wait.  The GPU
 * context stays usable afterwards. */
LNB_EXPORT int lnb_selftest_wait_timeout(long long wait_us);
/* The same for the factorization's device DAG (LNB_SCHED_DAG): the first
 * diagonal tile is never handed out, so every other task's wait runs out;
 * returns LNB_ETIMEOUT when the bound works. */
LNB_EXPORT int lnb_selftest_chol_wait_timeout(long long wait_us);

#ifdef __cplusplus
}
#endif
#endif /* LINOMPSS_B200_H */
