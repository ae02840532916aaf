/*
 * lnb_tasks.c -- the tile-task ABI (one BLAS/LAPACK operation on one tile).
 *
 * Replaces task_dpotrf (tasks_potrf.c:20-24), task_dtrsm (tasks_trsm.c:22-25),
 * task_dsyrk (tasks_syrk.c:19-21) and task_dgemm (task_gemm.c:55-58), which
 * the reference exports from libbblas and runs as OmpSs tasks.  Each call
 * here copies its tiles to the GPU, runs the corresponding kernel and copies
 * the result back, so an external caller that drives its own DAG over these
 * tasks gets GPU arithmetic with the same arguments.  The trailing `p`
 * (OmpSs priority) is accepted and ignored.
 */
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

#define EVEN(m) ((((int64_t)(m)) + 1) & ~(int64_t)1)

static int opt(const char *s, const char *allowed, char *out, const char *what)
{
    if (!s || !s[0] || !strchr(allowed, s[0])) return lnb_set_error(LNB_EINVAL, "bad %s option", what);
    *out = s[0];
    return 0;
}

static int put(double *d, int64_t ldd, const double *h, int64_t ldh, int64_t m, int64_t n, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    CK(cudaMemcpy2DAsync(d, ldd * sizeof(double), h, ldh * sizeof(double), m * sizeof(double), n,
                         cudaMemcpyHostToDevice, s), "tile in");
    return 0;
}
static int get(double *h, int64_t ldh, const double *d, int64_t ldd, int64_t m, int64_t n, cudaStream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    CK(cudaMemcpy2DAsync(h, ldh * sizeof(double), d, ldd * sizeof(double), m * sizeof(double), n,
                         cudaMemcpyDeviceToHost, s), "tile out");
    return 0;
}

int task_dpotrf(ompsslapack_t uplo, int n, double *A, int lda, int p)
{
    (void)p;
    char u = 0;
    int e = opt(uplo.s, "LU", &u, "uplo");
    if (e) return e;
    if (n < 0 || lda < (n > 1 ? n : 1) || n > 1024) return lnb_set_error(LNB_EINVAL, "potrf n=%d lda=%d", n, lda);
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = n;
    void *ws = lnb_ws(c, lnb_align256((size_t)ldd * n * sizeof(double)) + lnb_chol_f64_ws_bytes(n, n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = (double *)lnb_arena_take(&ar, (size_t)ldd * n * sizeof(double));
    double *dinv = (double *)lnb_arena_take(&ar, (size_t)((n + 31) / 32) * 1024 * sizeof(double));
    cudaStream_t s = c->main;
    double *tmp = NULL;
    if (u == 'U') {
        /* A = U^T U  <=>  A^T = L L^T with L = U^T: factor the transpose */
        tmp = (double *)malloc(sizeof(double) * (size_t)n * n);
        if (!tmp) return lnb_set_error(LNB_EINVAL, "host allocation");
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) tmp[i + (int64_t)j * n] = A[j + (int64_t)i * lda];
        e = put(dA, ldd, tmp, n, n, n, s);
    } else {
        e = put(dA, ldd, A, lda, n, n, s);
    }
    if (!e) e = (int)cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s) ? LNB_ECUDA : 0;
    if (!e) e = lnb_potrf_tile_f64(dA, ldd, n, 0, dinv, c->st, s);
    if (!e) e = get(u == 'U' ? tmp : A, u == 'U' ? n : lda, dA, ldd, n, n, s);
    int info = e ? e : lnb_status_read(c, s);
    if (u == 'U' && info >= 0) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i <= j; ++i) A[i + (int64_t)j * lda] = tmp[j + (int64_t)i * n];
    }
    free(tmp);
    return info;
}

int task_dgemm(ompssblas_t transa, ompssblas_t transb, int bm, int bn, int bk, double alpha, double *A,
               int lda, double *B, int ldb, double beta, double *C, int ldc, int p)
{
    (void)p;
    char ta = 0, tb = 0;
    int e;
    if ((e = opt(transa.s, "NT", &ta, "transa")) || (e = opt(transb.s, "NT", &tb, "transb"))) return e;
    if (bm < 0 || bn < 0 || bk < 0) return lnb_set_error(LNB_EINVAL, "gemm sizes");
    if (bm == 0 || bn == 0) return 0;
    const int64_t am = ta == 'N' ? bm : bk, an = ta == 'N' ? bk : bm;
    const int64_t bmr = tb == 'N' ? bk : bn, bnc = tb == 'N' ? bn : bk;
    if (lda < (am > 1 ? am : 1) || ldb < (bmr > 1 ? bmr : 1) || ldc < (bm > 1 ? bm : 1))
        return lnb_set_error(LNB_EINVAL, "gemm leading dimensions");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    /* device copies with even leading dimensions: every column starts on a
     * 16-byte boundary, as the kernel's 16-byte copies want */
    const int64_t lda_d = EVEN(am), ldb_d = EVEN(bmr), ldc_d = EVEN(bm);
    const size_t sa = lnb_align256((size_t)lda_d * (an ? an : 1) * 8), sb = lnb_align256((size_t)ldb_d * (bnc ? bnc : 1) * 8);
    const size_t sc = lnb_align256((size_t)ldc_d * bn * 8);
    void *ws = lnb_ws(c, sa + sb + sc + 1024);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, sa), *dB = lnb_arena_take(&ar, sb), *dC = lnb_arena_take(&ar, sc);
    cudaStream_t s = c->main;
    if ((e = put(dA, lda_d, A, lda, am, an, s)) || (e = put(dB, ldb_d, B, ldb, bmr, bnc, s)) ||
        (beta != 0.0 && (e = put(dC, ldc_d, C, ldc, bm, bn, s))))
        return e;
    CK(lnb_k_gemm_tri_f64(ta, tb, bm, bn, bk, alpha, dA, lda_d, dB, ldb_d, beta, dC, ldc_d, 0, s), "gemm");
    if ((e = get(C, ldc, dC, ldc_d, bm, bn, s))) return e;
    CK(cudaStreamSynchronize(s), "gemm sync");
    return 0;
}

int lnb_k_f32_to_f64(const float *X, int64_t ldx, int64_t m, int64_t k, double *D, int64_t ldd, cudaStream_t st);
int lnb_k_f64_to_f32(const double *D, int64_t ldd, int64_t m, int64_t k, float *X, int64_t ldx, cudaStream_t st);

/* C = alpha op(A) op(A)^T + beta C on triangle u of the host matrix C (FP64
 * or, with single != 0, FP32 host arrays computed in FP64 on the device) */
static int syrk_host(char u, char t, int n, int k, double alpha, const void *A, int lda, double beta, void *C,
                     int ldc, int single)
{
    if (n < 0 || k < 0) return lnb_set_error(LNB_EINVAL, "syrk sizes n = %d, k = %d", n, k);
    if (n == 0) return 0;
    const int64_t am = t == 'N' ? n : k, an = t == 'N' ? k : n;
    if (lda < (am > 1 ? am : 1) || ldc < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "syrk ld");
    if (!A || !C) return lnb_set_error(LNB_EINVAL, "syrk: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t lda_d = EVEN(am), ldc_d = EVEN(n);    /* 16-byte aligned device columns */
    const size_t sa = lnb_align256((size_t)lda_d * (an ? an : 1) * 8), sc = lnb_align256((size_t)ldc_d * n * 8);
    const size_t sa4 = single ? lnb_align256((size_t)am * (an ? an : 1) * 4) : 0;
    const size_t sc4 = single ? lnb_align256((size_t)n * n * 4) : 0;
    void *ws = lnb_ws(c, sa + sc + sa4 + sc4 + 1024);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, sa), *dC = lnb_arena_take(&ar, sc);
    float *fA = single ? (float *)lnb_arena_take(&ar, sa4) : NULL;
    float *fC = single ? (float *)lnb_arena_take(&ar, sc4) : NULL;
    cudaStream_t s = c->main;
    int e;
    if (!single) {
        if ((e = put(dA, lda_d, (const double *)A, lda, am, an, s)) ||
            (e = put(dC, ldc_d, (const double *)C, ldc, n, n, s)))
            return e;
    } else {
        if (am > 0 && an > 0) {
            CK(cudaMemcpy2DAsync(fA, (size_t)am * 4, A, (size_t)lda * 4, (size_t)am * 4, an, cudaMemcpyHostToDevice, s),
               "syrk A in");
            CK(lnb_k_f32_to_f64(fA, am, am, an, dA, lda_d, s), "widen A");
        }
        CK(cudaMemcpy2DAsync(fC, (size_t)n * 4, C, (size_t)ldc * 4, (size_t)n * 4, n, cudaMemcpyHostToDevice, s),
           "syrk C in");
        CK(lnb_k_f32_to_f64(fC, n, n, n, dC, ldc_d, s), "widen C");
    }
    CK(lnb_k_gemm_tri_f64(t == 'N' ? 'N' : 'T', t == 'N' ? 'T' : 'N', n, n, k, alpha, dA, lda_d, dA, lda_d, beta, dC,
                          ldc_d, u, s), "syrk");
    if (!single) {
        if ((e = get((double *)C, ldc, dC, ldc_d, n, n, s))) return e;
    } else {
        CK(lnb_k_f64_to_f32(dC, ldc_d, n, n, fC, n, s), "narrow C");
        CK(cudaMemcpy2DAsync(C, (size_t)ldc * 4, fC, (size_t)n * 4, (size_t)n * 4, n, cudaMemcpyDeviceToHost, s),
           "syrk C out");
    }
    CK(cudaStreamSynchronize(s), "syrk sync");
    return 0;
}

int ompss_dsyrk(ompssblas_t uplo, ompssblas_t trans, int b, int n, int k, double alpha, double *A, int lda,
                double beta, double *C, int ldc)
{
    char u = 0, t = 0;
    int e;
    if ((e = opt(uplo.s, "LU", &u, "uplo")) || (e = opt(trans.s, "NT", &t, "trans"))) return e;
    if (b <= 0) return lnb_set_error(LNB_EINVAL, "syrk tile size b = %d", b);
    return syrk_host(u, t, n, k, alpha, A, lda, beta, C, ldc, 0);
}

int ompss_ssyrk(ompssblas_t uplo, ompssblas_t trans, int b, int n, int k, float alpha, float *A, int lda,
                float beta, float *C, int ldc)
{
    char u = 0, t = 0;
    int e;
    if ((e = opt(uplo.s, "LU", &u, "uplo")) || (e = opt(trans.s, "NT", &t, "trans"))) return e;
    if (b <= 0) return lnb_set_error(LNB_EINVAL, "syrk tile size b = %d", b);
    return syrk_host(u, t, n, k, alpha, A, lda, beta, C, ldc, 1);
}

int task_dsyrk(ompssblas_t uplo, ompssblas_t trans, int n, int k, double alpha, double *A, int lda,
               double beta, double *C, int ldc, int p)
{
    (void)p;
    char u = 0, t = 0;
    int e;
    if ((e = opt(uplo.s, "LU", &u, "uplo")) || (e = opt(trans.s, "NT", &t, "trans"))) return e;
    return syrk_host(u, t, n, k, alpha, A, lda, beta, C, ldc, 0);
}

int task_dtrsm(ompssblas_t side, ompssblas_t uplo, ompssblas_t trans, ompssblas_t diag, int bm, int bn,
               double alpha, double *A, int lda, double *B, int ldb, int p)
{
    (void)p;
    char sd = 0, u = 0, t = 0, d = 0;
    int e;
    if ((e = opt(side.s, "LR", &sd, "side")) || (e = opt(uplo.s, "LU", &u, "uplo")) ||
        (e = opt(trans.s, "NT", &t, "trans")) || (e = opt(diag.s, "NU", &d, "diag")))
        return e;
    if (bm < 0 || bn < 0 || ldb < (bm > 1 ? bm : 1)) return lnb_set_error(LNB_EINVAL, "trsm sizes");
    const int64_t na = sd == 'L' ? bm : bn;
    if (lda < (na > 1 ? na : 1)) return lnb_set_error(LNB_EINVAL, "trsm lda");
    if (bm == 0 || bn == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const size_t sa = lnb_align256((size_t)na * na * 8), sb = lnb_align256((size_t)bm * bn * 8);
    void *ws = lnb_ws(c, sa + sb + lnb_trsm_f64_ws_bytes(na, sd == 'L' ? bn : bm) + 1024);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, sa), *dB = lnb_arena_take(&ar, sb);
    cudaStream_t s = c->main;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    if ((e = put(dA, na, A, lda, na, na, s))) return e;
    if (sd == 'L') {
        if ((e = put(dB, bm, B, ldb, bm, bn, s))) return e;
        if ((e = lnb_trsm_f64_run(c, u, t, d, bm, bn, alpha, dA, na, dB, bm, &ar, s, NULL))) return e;
        if ((e = get(B, ldb, dB, bm, bm, bn, s))) return e;
    } else {
        /* X op(A) = alpha B  <=>  op(A)^T X^T = alpha B^T */
        double *bt = (double *)malloc(sizeof(double) * (size_t)bm * bn);
        if (!bt) return lnb_set_error(LNB_EINVAL, "host allocation");
        for (int j = 0; j < bn; ++j)
            for (int i = 0; i < bm; ++i) bt[j + (int64_t)i * bn] = B[i + (int64_t)j * ldb];
        e = put(dB, bn, bt, bn, bn, bm, s);
        if (!e) e = lnb_trsm_f64_run(c, u, t == 'N' ? 'T' : 'N', d, bn, bm, alpha, dA, na, dB, bn, &ar, s, NULL);
        if (!e) e = get(bt, bn, dB, bn, bn, bm, s);
        if (!e) e = cudaStreamSynchronize(s) ? LNB_ECUDA : 0;
        if (!e)
            for (int j = 0; j < bn; ++j)
                for (int i = 0; i < bm; ++i) B[i + (int64_t)j * ldb] = bt[j + (int64_t)i * bn];
        free(bt);
        if (e) return e;
    }
    e = lnb_status_read(c, s);
    return e < 0 ? e : 0;
}

int lnb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double *dA, int lda,
                  const double *dB, int ldb, double beta, double *dC, int ldc, void *stream)
{
    if ((transa != 'N' && transa != 'T') || (transb != 'N' && transb != 'T'))
        return lnb_set_error(LNB_EINVAL, "dgemm options");
    if (m < 0 || n < 0 || k < 0) return lnb_set_error(LNB_EINVAL, "dgemm sizes");
    const int am = transa == 'N' ? m : k, br = transb == 'N' ? k : n;
    if (lda < (am > 1 ? am : 1) || ldb < (br > 1 ? br : 1) || ldc < (m > 1 ? m : 1))
        return lnb_set_error(LNB_EINVAL, "dgemm leading dimensions");
    if (m == 0 || n == 0) return 0;
    if (!dC || (k > 0 && (!dA || !dB))) return lnb_set_error(LNB_EINVAL, "dgemm: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    CK(lnb_k_gemm_tri_f64(transa, transb, m, n, k, alpha, dA, lda, dB, ldb, beta, dC, ldc, 0,
                          (cudaStream_t)stream), "dgemm");
    return 0;
}

int lnb_dsyrk_dev(char uplo, char trans, int n, int k, double alpha, const double *dA, int lda, double beta,
                  double *dC, int ldc, void *stream)
{
    if ((uplo != 'L' && uplo != 'U') || (trans != 'N' && trans != 'T'))
        return lnb_set_error(LNB_EINVAL, "dsyrk options");
    if (n < 0 || k < 0) return lnb_set_error(LNB_EINVAL, "dsyrk sizes");
    const int am = trans == 'N' ? n : k;
    if (lda < (am > 1 ? am : 1) || ldc < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "dsyrk leading dimensions");
    if (n == 0) return 0;
    if (!dC || (k > 0 && !dA)) return lnb_set_error(LNB_EINVAL, "dsyrk: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    CK(lnb_k_gemm_tri_f64(trans == 'N' ? 'N' : 'T', trans == 'N' ? 'T' : 'N', n, n, k, alpha, dA, lda, dA, lda, beta,
                          dC, ldc, uplo, (cudaStream_t)stream), "dsyrk");
    return 0;
}
