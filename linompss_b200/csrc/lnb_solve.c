/*
 * lnb_solve.c -- blocked triangular solves and the SPD solve (host C).
 *
 * bblas_dltrsm (bblas_trsm.h:116-202) walks block rows issuing one TRSM task
 * per diagonal block and one GEMM task per off-diagonal block; spdsolv_main
 * (spdsolv_main.c:10-20) runs it twice, L Y = B then L^T X = Y.  Here each
 * solve is one persistent DAG-walking launch (k_trsv.cu) after one launch
 * that inverts the 64 x 64 diagonal blocks; the forward and the backward
 * solve share the inverses.  With many right-hand sides the solve is instead
 * a sequence of DMMA GEMMs over 64-row blocks (trsm_gemm).
 */
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

#define TRSV_H 64

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

/* Two schedules for a solve: one persistent launch that walks the tile DAG,
 * or a sequence of DMMA GEMMs over 64-row blocks.  The DAG walk costs about
 * linearly in the right-hand sides; the GEMM sequence about 10 us per launch
 * plus full-rate tiles.  Measured on B200 (m = 1024 .. 16384), the GEMM
 * sequence wins from 128 - 256 columns on; auto switches at 192.  The GEMM
 * path needs at least TRSM_GEMM_MIN_NRHS columns (its workspace). */
#define TRSM_GEMM_MIN_NRHS 32
#define TRSM_GEMM_AUTO_NRHS 192

size_t lnb_trsm_f64_ws_bytes(int64_t n, int64_t nrhs)
{
    const int64_t nb = ceil_div(n, TRSV_H);
    return lnb_align256((size_t)nb * TRSV_H * TRSV_H * sizeof(double)) +
           lnb_align256((size_t)lnb_trsm_sync_ints(n, TRSV_H) * sizeof(int)) +
           (nrhs >= TRSM_GEMM_MIN_NRHS ? lnb_align256((size_t)TRSV_H * nrhs * sizeof(double)) : 0) + 512;
}

static int trsm_use_gemm(int64_t n, int64_t nrhs)
{
    static int mode = -2;
    if (mode == -2) {
        const char *e = getenv("LNB_TRSM_GEMM");    /* 0: always the DAG walk, 1: the GEMM path from 32 columns */
        mode = e ? atoi(e) : -1;
    }
    if (nrhs < TRSM_GEMM_MIN_NRHS || mode == 0) return 0;
    return mode == 1 || nrhs >= TRSM_GEMM_AUTO_NRHS;
}

/* op(T) X = alpha B by 64-row blocks in dependency order, the blocked solve of
 * bblas_dltrsm (bblas_trsm.h:119-160) with each TRSM task replaced by a
 * product with the inverted diagonal block:
 *     X_j = op(D_j) B_j                    (into tmp, then back into B_j)
 *     B_r = B_r - op(T)_{r,j} X_j          (every block row r still to come)
 * alpha enters through the first step: its diagonal product is scaled by
 * alpha and its update scales the rows still to come (beta = alpha), so
 * every later block already holds alpha B. */
static int trsm_gemm(char uplo, char trans, int64_t n, int64_t nrhs, double alpha, const double *T, int64_t ldt,
                     const double *dinv, double *B, int64_t ldb, double *tmp, cudaStream_t s)
{
    const int fwd = (uplo == 'L') == (trans == 'N');
    const int64_t nb = ceil_div(n, TRSV_H);
    for (int64_t q = 0; q < nb; ++q) {
        const int64_t j = fwd ? q : nb - 1 - q;
        const int64_t j0 = j * TRSV_H, jb = n - j0 < TRSV_H ? n - j0 : TRSV_H;
        CK(lnb_k_gemm_tri_f64(trans, 'N', jb, nrhs, jb, q == 0 ? alpha : 1.0, dinv + j * TRSV_H * TRSV_H, TRSV_H,
                              B + j0, ldb, 0.0, tmp, TRSV_H, 0, s), "diagonal block");
        CK(cudaMemcpy2DAsync(B + j0, (size_t)ldb * 8, tmp, TRSV_H * 8, (size_t)jb * 8, nrhs, cudaMemcpyDeviceToDevice,
                             s), "block back");
        const int64_t r0 = fwd ? j0 + jb : 0, nr = fwd ? n - j0 - jb : j0;
        if (nr <= 0) continue;
        /* op(T)_{r,j}: stored at rows r, columns j (below the diagonal block
         * for (L,N), above it for (U,N)); for trans 'T' it is the transpose of
         * the block at rows j, columns r (left of the diagonal block for
         * (L,T), right of it for (U,T)) */
        const double *Ap = trans == 'N' ? T + r0 + j0 * ldt : T + j0 + r0 * ldt;
        CK(lnb_k_gemm_tri_f64(trans, 'N', nr, nrhs, jb, -1.0, Ap, ldt, tmp, TRSV_H, q == 0 ? alpha : 1.0, B + r0, ldb,
                              0, s), "update");
    }
    return 0;
}

/* op(T) X = alpha B with T triangular (uplo as stored), left side */
int lnb_trsm_f64_run(lnb_ctx *c, char uplo, char trans, char diag, int64_t n, int64_t nrhs,
                     double alpha, const double *dT, int64_t ldt, double *dB, int64_t ldb,
                     lnb_arena *ar, cudaStream_t s, const double *dinv_given)
{
    if (n <= 0 || nrhs <= 0) return 0;
    if (alpha == 0.0) {                /* BLAS: B = 0, T not read */
        CK(cudaMemset2DAsync(dB, (size_t)ldb * 8, 0, (size_t)n * 8, nrhs, s), "zero");
        return 0;
    }
    const int64_t nb = ceil_div(n, TRSV_H);
    double *dinv = (double *)dinv_given;
    if (!dinv) {
        dinv = (double *)lnb_arena_take(ar, (size_t)nb * TRSV_H * TRSV_H * sizeof(double));
        if (!dinv) return lnb_set_error(LNB_ENOMEM, "trsm workspace");
        CK(lnb_k_trtri_blocks_f64(dT, ldt, n, TRSV_H, uplo, diag == 'U', dinv, s), "trtri");
    }
    if (trsm_use_gemm(n, nrhs)) {
        double *tmp = (double *)lnb_arena_take(ar, (size_t)TRSV_H * nrhs * sizeof(double));
        if (!tmp) return lnb_set_error(LNB_ENOMEM, "trsm workspace");
        return trsm_gemm(uplo, trans, n, nrhs, alpha, dT, ldt, dinv, dB, ldb, tmp, s);
    }
    int *sync = (int *)lnb_arena_take(ar, (size_t)lnb_trsm_sync_ints(n, TRSV_H) * sizeof(int));
    if (!sync) return lnb_set_error(LNB_ENOMEM, "trsm sync workspace");
    CK(lnb_k_trsm_left_f64(uplo, trans, n, nrhs, alpha, dT, ldt, dinv, TRSV_H, dB, ldb, sync, c->st,
                           lnb_wait_ns(), 0, s), "trsm dag");
    return 0;
}

int lnb_selftest_wait_timeout(long long wait_us)
{
    /* 1024 x 1024 identity, 1 rhs.  The ticket starts at 1, so no CTA walks
     * the diagonal chain, and the off-band update items wait on solution
     * blocks that nothing publishes. */
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t n = 1024;
    void *ws = lnb_ws(c, lnb_align256(n * n * 8) + lnb_align256(n * 8) + lnb_trsm_f64_ws_bytes(n, 1));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *T = lnb_arena_take(&ar, n * n * 8), *B = lnb_arena_take(&ar, n * 8);
    double *dinv = lnb_arena_take(&ar, (size_t)ceil_div(n, TRSV_H) * TRSV_H * TRSV_H * 8);
    int *sync = lnb_arena_take(&ar, (size_t)lnb_trsm_sync_ints(n, TRSV_H) * sizeof(int));
    cudaStream_t s = c->main;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(cudaMemsetAsync(T, 0, n * n * 8, s), "zero");
    CK(cudaMemsetAsync(B, 0, n * 8, s), "zero");
    CK(lnb_k_trtri_blocks_f64(T, n, n, TRSV_H, 'L', 1, dinv, s), "trtri");
    CK(lnb_k_trsm_left_f64('L', 'N', n, 1, 1.0, T, n, dinv, TRSV_H, B, n, sync, c->st,
                           (wait_us > 0 ? wait_us : 1000) * 1000LL, 1, s), "trsm dag");
    return lnb_status_read(c, s);
}

static int opt_char(ompssblas_t o, const char *allowed, char *out, const char *what)
{
    if (!o.s || !o.s[0] || !strchr(allowed, o.s[0]))
        return lnb_set_error(LNB_EINVAL, "bad %s option", what);
    *out = o.s[0];
    return 0;
}

/* ---- device-pointer entry points ---------------------------------------- */
int lnb_dtrsm_dev(char uplo, char trans, char diag, int m, int n, double alpha, const double *dA,
                  int lda, double *dB, int ldb, void *stream)
{
    if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1))
        return lnb_set_error(LNB_EINVAL, "dtrsm sizes m=%d n=%d lda=%d ldb=%d", m, n, lda, ldb);
    if ((uplo != 'L' && uplo != 'U') || (trans != 'N' && trans != 'T') || (diag != 'N' && diag != 'U'))
        return lnb_set_error(LNB_EINVAL, "dtrsm options");
    if (m == 0 || n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, lnb_trsm_f64_ws_bytes(m, n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    return lnb_trsm_f64_run(c, uplo, trans, diag, m, n, alpha, dA, lda, dB, ldb, &ar, s, NULL);
}

int lnb_dsymv_dev(int n, int nrhs, const double *dA, int lda, const double *dX, double *dY, void *stream)
{
    if (n < 0 || nrhs < 0 || lda < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "dsymv sizes");
    if (n == 0 || nrhs == 0) return 0;
    if (!dA || !dX || !dY) return lnb_set_error(LNB_EINVAL, "dsymv: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    CK(lnb_k_symv_lower_f64(n, nrhs, dA, lda, dX, dY, 0, (cudaStream_t)stream), "dsymv");
    return 0;
}

int lnb_dpotrs_dev(int n, int nrhs, const double *dL, int lda, double *dB, int ldb, char which,
                   void *stream)
{
    if (n < 0 || nrhs < 0 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "potrs sizes");
    if (which != 'N' && which != 'T' && which != 'B') return lnb_set_error(LNB_EINVAL, "potrs which");
    if (n == 0 || nrhs == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, 2 * lnb_trsm_f64_ws_bytes(n, nrhs));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    const int64_t nb = ceil_div(n, TRSV_H);
    double *dinv = (double *)lnb_arena_take(&ar, (size_t)nb * TRSV_H * TRSV_H * sizeof(double));
    CK(lnb_k_trtri_blocks_f64(dL, lda, n, TRSV_H, 'L', 0, dinv, s), "trtri");
    int e = 0;
    if (which == 'N' || which == 'B')
        e = lnb_trsm_f64_run(c, 'L', 'N', 'N', n, nrhs, 1.0, dL, lda, dB, ldb, &ar, s, dinv);
    if (!e && (which == 'T' || which == 'B'))
        e = lnb_trsm_f64_run(c, 'L', 'T', 'N', n, nrhs, 1.0, dL, lda, dB, ldb, &ar, s, dinv);
    return e;
}

int lnb_dposv_dev(int n, int nrhs, int b, double *dA, int lda, double *dB, int ldb, int *info_dev,
                  void *stream)
{
    if (n < 0 || nrhs < 0 || b <= 0 || b > 1024 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "posv arguments");
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t nb = ceil_div(n, TRSV_H);
    void *ws = lnb_ws(c, lnb_chol_f64_ws_bytes(n, b) + 2 * lnb_trsm_f64_ws_bytes(n, nrhs));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    double *dinv = NULL;
    int e = lnb_chol_f64_run_w(c, n, b, dA, lda, &ar, s, NULL, 0, &dinv);
    if (e) return e;
    if (nrhs > 0) {
        /* the device DAG leaves the 64 x 64 diagonal-block inverses the solves use */
        if (!dinv) {
            dinv = (double *)lnb_arena_take(&ar, (size_t)nb * TRSV_H * TRSV_H * sizeof(double));
            if (!dinv) return lnb_set_error(LNB_ENOMEM, "posv workspace");
            CK(lnb_k_trtri_blocks_f64(dA, lda, n, TRSV_H, 'L', 0, dinv, s), "trtri");
        }
        if ((e = lnb_trsm_f64_run(c, 'L', 'N', 'N', n, nrhs, 1.0, dA, lda, dB, ldb, &ar, s, dinv))) return e;
        if ((e = lnb_trsm_f64_run(c, 'L', 'T', 'N', n, nrhs, 1.0, dA, lda, dB, ldb, &ar, s, dinv))) return e;
    }
    if (info_dev)
        CK(cudaMemcpyAsync(info_dev, &c->st->info, sizeof(int), cudaMemcpyDeviceToDevice, s), "info");
    return 0;
}

/* ---- host entry points ---------------------------------------------------- */
static inline int64_t ld_dev(int64_t n) { return (n + 7) & ~(int64_t)7; }

int dspdsolv_main(int m, int nrhs, int b, double *A, double *B)
{
    if (m < 0 || nrhs < 0 || b <= 0 || b > 1024) return lnb_set_error(LNB_EINVAL, "spdsolv arguments");
    if (m == 0) return 0;
    if (!A || (nrhs > 0 && !B)) return lnb_set_error(LNB_EINVAL, "NULL matrix");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ld_dev(m);
    const size_t abytes = (size_t)ldd * m * sizeof(double), bbytes = (size_t)ldd * (nrhs ? nrhs : 1) * sizeof(double);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_align256(bbytes) + lnb_chol_f64_ws_bytes(m, b) +
                             2 * lnb_trsm_f64_ws_bytes(m, nrhs));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = (double *)lnb_arena_take(&ar, abytes);
    double *dB = (double *)lnb_arena_take(&ar, bbytes);
    cudaStream_t s = c->main;
    /* lower block-columns of A, all of B */
    for (int64_t c0 = 0; c0 < m; c0 += b) {
        int64_t w = m - c0 < b ? m - c0 : b;
        CK(cudaMemcpy2DAsync(dA + c0 + c0 * ldd, ldd * sizeof(double), A + c0 + c0 * (int64_t)m,
                             (size_t)m * sizeof(double), (size_t)(m - c0) * sizeof(double), w,
                             cudaMemcpyHostToDevice, s), "A in");
    }
    if (nrhs > 0)
        CK(cudaMemcpy2DAsync(dB, ldd * sizeof(double), B, (size_t)m * sizeof(double),
                             (size_t)m * sizeof(double), nrhs, cudaMemcpyHostToDevice, s), "B in");
    const int pinned = lnb_host_is_pinned(A);
    double *dinv = NULL;
    int e = lnb_chol_f64_run_w(c, m, b, dA, ldd, &ar, s, pinned ? A : NULL, m, &dinv);
    if (e) return e;
    if (nrhs > 0) {
        if (!dinv) {
            const int64_t nb = ceil_div(m, TRSV_H);
            dinv = (double *)lnb_arena_take(&ar, (size_t)nb * TRSV_H * TRSV_H * sizeof(double));
            if (!dinv) return lnb_set_error(LNB_ENOMEM, "spdsolv workspace");
            CK(lnb_k_trtri_blocks_f64(dA, ldd, m, TRSV_H, 'L', 0, dinv, s), "trtri");
        }
        if ((e = lnb_trsm_f64_run(c, 'L', 'N', 'N', m, nrhs, 1.0, dA, ldd, dB, ldd, &ar, s, dinv))) return e;
        if ((e = lnb_trsm_f64_run(c, 'L', 'T', 'N', m, nrhs, 1.0, dA, ldd, dB, ldd, &ar, s, dinv))) return e;
        CK(cudaMemcpy2DAsync(B, (size_t)m * sizeof(double), dB, ldd * sizeof(double),
                             (size_t)m * sizeof(double), nrhs, cudaMemcpyDeviceToHost, s), "X out");
    }
    if (!pinned)
        for (int64_t c0 = 0; c0 < m; c0 += b) {
            int64_t w = m - c0 < b ? m - c0 : b;
            CK(cudaMemcpy2DAsync(A + c0 + c0 * (int64_t)m, (size_t)m * sizeof(double), dA + c0 + c0 * ldd,
                                 ldd * sizeof(double), (size_t)(m - c0) * sizeof(double), w,
                                 cudaMemcpyDeviceToHost, s), "L out");
        }
    return lnb_status_read(c, s);
}

int ompss_dtrsm(ompssblas_t side, ompssblas_t uplo, ompssblas_t trans, ompssblas_t diag, int m, int n,
                int b, double alpha, double *A, int lda, double *B, int ldb)
{
    char cs = 0, cu = 0, ct = 0, cd = 0;
    int e;
    if ((e = opt_char(side, "LR", &cs, "side")) || (e = opt_char(uplo, "LU", &cu, "uplo")) ||
        (e = opt_char(trans, "NT", &ct, "trans")) || (e = opt_char(diag, "NU", &cd, "diag")))
        return e;
    (void)b;
    if (cs != 'L') return lnb_set_error(LNB_EINVAL, "rtrsm: not implemented (as in trsm_main.c:13)");
    if (m < 0 || n < 0 || lda < (m > 1 ? m : 1) || ldb < (m > 1 ? m : 1))
        return lnb_set_error(LNB_EINVAL, "dtrsm sizes");
    if (m == 0 || n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ld_dev(m);
    const size_t abytes = (size_t)ldd * m * sizeof(double), bbytes = (size_t)ldd * n * sizeof(double);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_align256(bbytes) + lnb_trsm_f64_ws_bytes(m, n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = (double *)lnb_arena_take(&ar, abytes);
    double *dB = (double *)lnb_arena_take(&ar, bbytes);
    cudaStream_t s = c->main;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(cudaMemcpy2DAsync(dA, ldd * sizeof(double), A, (size_t)lda * sizeof(double), (size_t)m * sizeof(double),
                         m, cudaMemcpyHostToDevice, s), "A in");
    CK(cudaMemcpy2DAsync(dB, ldd * sizeof(double), B, (size_t)ldb * sizeof(double), (size_t)m * sizeof(double),
                         n, cudaMemcpyHostToDevice, s), "B in");
    if ((e = lnb_trsm_f64_run(c, cu, ct, cd, m, n, alpha, dA, ldd, dB, ldd, &ar, s, NULL))) return e;
    CK(cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(double), dB, ldd * sizeof(double), (size_t)m * sizeof(double),
                         n, cudaMemcpyDeviceToHost, s), "B out");
    e = lnb_status_read(c, s);
    return e < 0 ? e : 0;
}
