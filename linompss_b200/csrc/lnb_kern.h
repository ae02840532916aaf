/*
 * lnb_kern.h -- internal C ABI between the host-side C drivers and the CUDA
 * kernel launchers (the "thin C-ABI layer").  Not installed; the public ABI
 * is include/linompss_b200.h.
 *
 * Every launcher enqueues on `stream` and returns a cudaError_t value
 * (0 = cudaSuccess) as int.  All matrices are column-major with 64-bit
 * leading dimensions.
 */
#ifndef LNB_KERN_H
#define LNB_KERN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *lnb_stream_t;

/* Device-side status word shared by the kernels of one call. */
typedef struct {
    int info;          /* first non-positive pivot (1-based, global row), 0 if none */
    int timeout;       /* set to a site code when a bounded wait ran out */
    int timeout_item;  /* work item that gave up */
    int pad;
} lnb_status_t;

/* ---- FP64 factorization kernels (k_chol_f64.cu) ------------------------- */
/* Factor the bs x bs diagonal tile at A (in place, lower).  If dinv != NULL,
 * also writes the inverses of its 32 x 32 diagonal blocks (ceil(bs/32)
 * blocks, each 32 x 32 column-major, unit-padded past bs).  row0 is the
 * tile's global row offset (for info). */
int lnb_k_potrf_f64(double *A, int64_t lda, int bs, int64_t row0, double *dinv,
                    lnb_status_t *st, lnb_stream_t s);
/* B (m x bs) <- B * L^-T with L the bs x bs lower tile at L (ld lda) and
 * dinv its 32-block inverses from lnb_k_potrf_f64. */
int lnb_k_trsm_rlt_f64(const double *L, int64_t lda, const double *dinv, double *B,
                       int64_t ldb, int64_t m, int bs, lnb_stream_t s);
/* C[r,c] -= sum_k P[r,k] P[c,k] for r >= c, 0 <= r < nrows, c0 <= c < c1,
 * k < kdim.  P and C are both indexed from the trailing matrix's origin. */
int lnb_k_syrk_lower_f64(const double *P, int64_t ldp, double *C, int64_t ldc,
                         int64_t nrows, int64_t c0, int64_t c1, int kdim, lnb_stream_t s);
/* Generic C = alpha op(A) op(B) + beta C on device memory (tile-task ABI),
 * restricted to the triangle tri ('L' or 'U') of C; tri = 0: full. */
int lnb_k_gemm_tri_f64(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                       const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                       double *C, int64_t ldc, char tri, lnb_stream_t s);

/* Whole FP64 factorization as one persistent launch walking the tile DAG on
 * the device (k_chol_dag.cu): 64 x 64 tiles, A in place (lower), W receives
 * the inverses of the diagonal tiles (64 x 64 column-major each, identity past
 * n), sync lnb_chol_dag_ints(n) ints of scratch (zeroed by the launcher).
 * ticket0 > 0 only in the wait self-test. */
int64_t lnb_chol_dag_ints(int64_t n);
int64_t lnb_chol_dag_w_doubles(int64_t n);
int lnb_k_chol_dag_f64(double *A, int64_t lda, int64_t n, double *W, int *sync, lnb_status_t *st,
                       long long wait_ns, int sms, int ticket0, lnb_stream_t s);

/* ---- triangular solves (k_trsv.cu) --------------------------------------- */
/* Inverses of the h x h diagonal blocks of T: dinv block q (h x h,
 * column-major) is (T[qh:qh+h, qh:qh+h])^-1 for the triangle `uplo` of T,
 * unit diagonal if unit != 0; padded with the identity past n.  h = 64. */
int lnb_k_trtri_blocks_f64(const double *T, int64_t ldt, int64_t n, int h, char uplo, int unit,
                           double *dinv, lnb_stream_t s);
/* Solve op(T) X = alpha B in place (B n x nrhs, ld ldb) with the block
 * inverses from lnb_k_trtri_blocks_f64.  uplo/trans describe T as stored.
 * One persistent launch walks the solve's tile DAG; every dependency wait is
 * bounded by wait_ns of device time (st->timeout set on expiry).
 * sync: device scratch of lnb_trsm_sync_ints(n, h) ints (zeroed here). */
int64_t lnb_trsm_sync_ints(int64_t n, int h);
/* ticket0: first work item handed out (0; > 0 only in the wait self-test,
 * where skipping item 0 leaves a dependency that is never satisfied). */
int lnb_k_trsm_left_f64(char uplo, char trans, int64_t n, int64_t nrhs, double alpha,
                        const double *T, int64_t ldt, const double *dinv, int h, double *B,
                        int64_t ldb, int *sync, lnb_status_t *st, long long wait_ns,
                        int ticket0, lnb_stream_t s);

/* Few right-hand sides (nrhs <= 8): the same solve as one launch built
 * around the diagonal chain (k_trsv_chain.cu).  sync as above, zeroed by the
 * caller; alpha already applied. */
int lnb_k_trsm_chain_f64(char uplo, char trans, int64_t n, int64_t nrhs, const double *T, int64_t ldt,
                         const double *dinv, double *B, int64_t ldb, int *sync, lnb_status_t *st,
                         long long wait_ns, lnb_stream_t s);
int lnb_k_trsm_chain_f32(char uplo, char trans, int64_t n, int64_t nrhs, const float *T, int64_t ldt,
                         const float *dinv, double *B, int64_t ldb, int *sync, lnb_status_t *st,
                         long long wait_ns, lnb_stream_t s);

/* ---- FP32-storage factorization kernels (k_chol_f32.cu) ------------------ */
int lnb_k_potrf_f32(float *A, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                    lnb_stream_t s);
int lnb_k_trsm_rlt_f32(const float *L, int64_t lda, const float *dinv, float *B, int64_t ldb, int64_t m,
                       int bs, lnb_stream_t s);
/* the same solve, also writing the K-major TF32 operand copies of the result
 * (hi = rna_tf32(x); lo = x - hi when lo != NULL), rows of kpad elements */
int lnb_k_trsm_rlt_prep_f32(const float *L, int64_t lda, const float *dinv, float *B, int64_t ldb, int64_t m,
                            int bs, float *hi, float *lo, int kpad, lnb_stream_t s);
int lnb_k_syrk_lower_f32_simt(const float *P, int64_t ldp, float *C, int64_t ldc, int64_t nrows,
                              int64_t c0, int64_t c1, int kdim, lnb_stream_t s);
/* K-major BF16 operand copy of a solved panel X (m x kb, ld ldx) with
 * per-128-row power-of-two scales (the TF32 copies come from the panel solve) */
int lnb_k_prep_bf16(const float *X, int64_t ldx, int64_t m, int kb, int kpad, float *scale, void *out,
                    lnb_stream_t s);
/* A32 = lower(S A S) in FP32 with S = diag(1/sqrt(a_ii)) (S = I if !equilibrate);
 * rsum (may be NULL, else zeroed by the caller) gains the row sums of |A| of
 * the symmetric A whose lower triangle is given, for its infinity norm */
int lnb_k_lower_to_f32(const double *A, int64_t lda, int64_t n, int equilibrate, double *s_out,
                       float *A32, int64_t ld32, double *rsum, lnb_stream_t s);
/* A32 columns [c0, c1), rows >= column: lower(S A S) in FP32, S given; rsum as
 * above, for the elements of these columns */
int lnb_k_lower_to_f32_cols(const double *A, int64_t lda, int64_t n, int64_t c0, int64_t c1, const double *S,
                            float *A32, int64_t ld32, double *rsum, lnb_stream_t s);
/* s[i] = 1/sqrt(a[i]) (1 when !on or a[i] <= 0) from a packed diagonal; s may alias a */
int lnb_k_equil_scale_vec(const double *a, int64_t n, int on, double *s, lnb_stream_t st);
/* tensor-core lower update (k_tc_update.cu); mode 0 TF32x3, 1 TF32, 2 BF16.
 * hi/lo: K-major operand copies (prow rows, row stride kstride, first kdim K
 * columns used); C FP32 column-major. */
int lnb_k_tc_syrk_lower(int mode, const void *hi, const void *lo, int64_t kstride, int64_t prow, float *C,
                        int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim, const float *scale,
                        lnb_status_t *st, long long wait_ns, lnb_stream_t s);

/* FP32-stored triangular factor, FP64 right-hand sides and arithmetic; the block
 * inverses are stored in FP32 (computed in FP64) */
int lnb_k_trtri_blocks_f32(const float *T, int64_t ldt, int64_t n, int h, char uplo, int unit, float *dinv,
                           lnb_stream_t s);
int lnb_k_trsm_left_f32(char uplo, char trans, int64_t n, int64_t nrhs, double alpha, const float *T,
                        int64_t ldt, const float *dinv, int h, double *B, int64_t ldb, int *sync,
                        lnb_status_t *st, long long wait_ns, int ticket0, lnb_stream_t s);

/* ---- symmetric products and refinement vectors (k_symv.cu) --------------- */
/* Y = A X for symmetric A given by its lower triangle (FP64, column-major),
 * X, Y n x nrhs (ld n); Y is overwritten.  absval != 0 uses |A| (row sums of
 * |A| with X = ones give ||A||_inf). */
int lnb_k_symv_lower_f64(int64_t n, int64_t nrhs, const double *A, int64_t lda, const double *X, double *Y,
                         int absval, lnb_stream_t s);
/* R = B - Y  and per-column max |R| into rmax[nrhs] (R may alias Y) */
int lnb_k_resid_f64(int64_t n, int64_t nrhs, const double *B, int64_t ldb, const double *Y, double *R,
                    double *rmax, lnb_stream_t s);
/* per-column max |X| into out[nrhs] */
int lnb_k_colmax_f64(int64_t n, int64_t nrhs, const double *X, int64_t ldx, double *out, lnb_stream_t s);
/* Z = diag(sc) R   (sc may be NULL: copy) */
int lnb_k_scale_rows_f64(int64_t n, int64_t nrhs, const double *sc, const double *R, double *Z, lnb_stream_t s);
/* X += diag(sc) Z */
int lnb_k_axpy_scaled_f64(int64_t n, int64_t nrhs, const double *sc, const double *Z, double *X, int64_t ldx,
                          lnb_stream_t s);

/* launch accounting (lnb_runtime.c), called by every launcher */
void lnb_prof_count(int kernels);

/* ---- FP64 vector kernels (k_blas1.cu); reductions are deterministic ------- */
int64_t lnb_gemv_part_doubles(int64_t m, int64_t n);
int64_t lnb_dot_part_doubles(int64_t n);
/* y = alpha A x + beta yin (A m x n).  If dot_out: *dot_out = <y, w>.
 * part: lnb_gemv_part_doubles(m, n) doubles; dpart: lnb_dot_part_doubles(m). */
int lnb_k_gemv_f64(int64_t m, int64_t n, double alpha, const double *A, int64_t lda, const double *x,
                   double beta, const double *yin, double *y, const double *w, double *dot_out,
                   double *part, double *dpart, lnb_stream_t s);
int lnb_k_dot_f64(int64_t n, const double *x, const double *y, double *out, double *dpart,
                  lnb_stream_t s);
/* f = num/den; x += f p; r -= f tmp; *rr_out = <r, r> */
int lnb_k_cg_xr_f64(int64_t n, const double *num, const double *den, const double *p,
                    const double *tmp, double *x, double *r, double *rr_out, double *dpart,
                    lnb_stream_t s);
/* mode 0: p = 2 r (the reference's executed update); mode 1: p = r + (num/den) p */
int lnb_k_cg_p_f64(int64_t n, int mode, const double *num, const double *den, const double *r,
                   double *p, lnb_stream_t s);
int lnb_k_axpy3_f64(int64_t n, double a, const double *x, const double *y, double *z, lnb_stream_t s);

#ifdef __cplusplus
}
#endif
#endif
