/*
 * lnb_lu.c -- tile LU with partial pivoting and the general solve (host C).
 *
 * Replaces ompss_dgetrf / ompss_sgetrf and their _ll twins (ompss_lu.h:15-21,
 * dlu_main lu_main.c:5-27, dlull_main lull_main.c) and dgensolv_main /
 * sgensolv_main (gensolv_main.c:10-25).
 *
 * The reference factors b-wide panels with LAPACK dgetrf over every row below
 * (so its pivots are LAPACK's), then swaps the other block columns and updates
 * those on the right with a unit-lower TRSM and a GEMM.  Here the same
 * factorization is blocked for the GPU at two levels:
 *   * outer blocks of 256 columns: once a block is factored, its swaps go to
 *     every other column, its rows of U come from one blocked TRSM
 *     (lnb_trsm_f64_run, unit lower), and the rest of the matrix takes one
 *     DMMA GEMM of depth 256;
 *   * inside a block, panels of up to 32 columns are factored in shared memory
 *     by one thread-block cluster (k_lu.cu), and the block's remaining columns
 *     take the panel's swaps, a small unit-lower solve and a GEMM.
 * Partial pivoting over all rows below gives LAPACK's pivot sequence whatever
 * the blocking, so the user's b only shapes the pivot indices returned: the
 * reference leaves each b-wide panel's pivots as dgetrf returned them for the
 * panel (1-based, relative to the panel's first row), and so does this file.
 * Where the reference's swaps are incomplete (a ragged last panel swaps only
 * dimC columns of the earlier blocks, lu_main.c TASK_LASWP; gensolv applies
 * panel i's swaps from row b instead of row i) no swap happens on the matrices
 * it generates (a +100 diagonal), and here every swap is applied in full.
 */
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

#define LU_BO 256

int lnb_lu_panel_width(int64_t rows);
int lnb_k_lu_panel_f64(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int *piv, lnb_status_t *st,
                       cudaStream_t s);
int lnb_k_laswp_f64(double *A, int64_t lda, int64_t k0, int64_t k1, const int *piv, int64_t a0, int64_t a1,
                    int64_t b0, int64_t b1, cudaStream_t s);
int lnb_k_lu_trsm_unit_f64(double *A, int64_t lda, int64_t c0, int nb, int64_t j0, int64_t j1, cudaStream_t s);
int lnb_k_f32_to_f64(const float *X, int64_t ldx, int64_t m, int64_t k, double *D, int64_t ldd, cudaStream_t st);
int lnb_k_f64_to_f32(const double *D, int64_t ldd, int64_t m, int64_t k, float *X, int64_t ldx, cudaStream_t st);

static size_t getrf_ws_bytes(int64_t n) { return lnb_trsm_f64_ws_bytes(LU_BO, n) + 1024; }

/* P A = L U of dA (m x n) in place; dpiv: min(m, n) LAPACK pivots (1-based,
 * global rows).  An exactly zero pivot sets st->info (its 1-based column). */
static int getrf_run(lnb_ctx *c, int64_t m, int64_t n, double *dA, int64_t lda, int *dpiv, lnb_arena *ar,
                     cudaStream_t s)
{
    const int64_t mn = m < n ? m : n;
    if (mn <= 0) return 0;
    if (!lnb_lu_panel_width(m))
        return lnb_set_error(LNB_ETOOBIG, "getrf: %lld rows exceed a panel cluster's shared memory", (long long)m);
    for (int64_t o0 = 0; o0 < mn; o0 += LU_BO) {
        const int64_t ob = mn - o0 < LU_BO ? mn - o0 : LU_BO, oe = o0 + ob;
        for (int64_t c0 = o0; c0 < oe;) {
            int nb = lnb_lu_panel_width(m - c0);
            if (nb > oe - c0) nb = (int)(oe - c0);
            CK(lnb_k_lu_panel_f64(dA, lda, m, c0, nb, dpiv, c->st, s), "lu panel");
            CK(lnb_k_laswp_f64(dA, lda, c0, c0 + nb, dpiv, o0, c0, c0 + nb, oe, s), "panel swaps");
            if (c0 + nb < oe) {
                CK(lnb_k_lu_trsm_unit_f64(dA, lda, c0, nb, c0 + nb, oe, s), "panel solve");
                if (m > c0 + nb)
                    CK(lnb_k_gemm_tri_f64('N', 'N', m - c0 - nb, oe - c0 - nb, nb, -1.0, dA + (c0 + nb) + c0 * lda,
                                          lda, dA + c0 + (c0 + nb) * lda, lda, 1.0,
                                          dA + (c0 + nb) + (c0 + nb) * lda, lda, 0, s), "panel update");
            }
            c0 += nb;
        }
        CK(lnb_k_laswp_f64(dA, lda, o0, oe, dpiv, 0, o0, oe, n, s), "block swaps");
        if (oe < n) {
            lnb_arena a2 = *ar;
            const int e = lnb_trsm_f64_run(c, 'L', 'N', 'U', ob, n - oe, 1.0, dA + o0 + o0 * lda, lda,
                                           dA + o0 + oe * lda, lda, &a2, s, NULL);
            if (e) return e;
            if (m > oe)
                CK(lnb_k_gemm_tri_f64('N', 'N', m - oe, n - oe, ob, -1.0, dA + oe + o0 * lda, lda, dA + o0 + oe * lda,
                                      lda, 1.0, dA + oe + oe * lda, lda, 0, s), "trailing update");
        }
    }
    return 0;
}

/* X = A^-1 B from getrf's factors: B's rows take the pivots, then the unit
 * lower and the upper solve (gensolv_main.c:15-22) */
static int getrs_run(lnb_ctx *c, int64_t n, int64_t nrhs, const double *dLU, int64_t lda, const int *dpiv,
                     double *dB, int64_t ldb, lnb_arena *ar, cudaStream_t s)
{
    if (n <= 0 || nrhs <= 0) return 0;
    CK(lnb_k_laswp_f64(dB, ldb, 0, n, dpiv, 0, nrhs, 0, 0, s), "rhs swaps");
    lnb_arena a2 = *ar;
    int e = lnb_trsm_f64_run(c, 'L', 'N', 'U', n, nrhs, 1.0, dLU, lda, dB, ldb, &a2, s, NULL);
    if (e) return e;
    a2 = *ar;
    return lnb_trsm_f64_run(c, 'U', 'N', 'N', n, nrhs, 1.0, dLU, lda, dB, ldb, &a2, s, NULL);
}

static inline int64_t ld_dev(int64_t m) { return (m + 7) & ~(int64_t)7; }

/* host matrix (m x n, ld, FP64 or FP32) -> device FP64 (ld ldd) */
static int mat_in(double *d, int64_t ldd, const void *h, int64_t ld, int64_t m, int64_t n, float *f32,
                  cudaStream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    if (!f32) {
        CK(cudaMemcpy2DAsync(d, (size_t)ldd * 8, h, (size_t)ld * 8, (size_t)m * 8, n, cudaMemcpyHostToDevice, s),
           "matrix in");
    } else {
        CK(cudaMemcpy2DAsync(f32, (size_t)m * 4, h, (size_t)ld * 4, (size_t)m * 4, n, cudaMemcpyHostToDevice, s),
           "matrix in");
        CK(lnb_k_f32_to_f64(f32, m, m, n, d, ldd, s), "widen");
    }
    return 0;
}
static int mat_out(void *h, int64_t ld, const double *d, int64_t ldd, int64_t m, int64_t n, float *f32,
                   cudaStream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    if (!f32) {
        CK(cudaMemcpy2DAsync(h, (size_t)ld * 8, d, (size_t)ldd * 8, (size_t)m * 8, n, cudaMemcpyDeviceToHost, s),
           "matrix out");
    } else {
        CK(lnb_k_f64_to_f32(d, ldd, m, n, f32, m, s), "narrow");
        CK(cudaMemcpy2DAsync(h, (size_t)ld * 4, f32, (size_t)m * 4, (size_t)m * 4, n, cudaMemcpyDeviceToHost, s),
           "matrix out");
    }
    return 0;
}

static int getrf_host(int m, int n, int b, void *A, int lda, int *IPIV, int single)
{
    if (m < 0 || n < 0 || b <= 0 || lda < (m > 1 ? m : 1))
        return lnb_set_error(LNB_EINVAL, "getrf arguments m=%d n=%d b=%d lda=%d", m, n, b, lda);
    const int mn = m < n ? m : n;
    if (mn == 0) return 0;
    if (!A || !IPIV) return lnb_set_error(LNB_EINVAL, "getrf: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ld_dev(m);
    const size_t abytes = (size_t)ldd * n * 8, pbytes = (size_t)mn * 4, fbytes = single ? (size_t)m * n * 4 : 0;
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_align256(pbytes) + lnb_align256(fbytes) + getrf_ws_bytes(n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, abytes);
    int *dpiv = lnb_arena_take(&ar, pbytes);
    float *f32 = single ? lnb_arena_take(&ar, fbytes) : NULL;
    cudaStream_t s = c->main;
    int e;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    if ((e = mat_in(dA, ldd, A, lda, m, n, f32, s))) return e;
    if ((e = getrf_run(c, m, n, dA, ldd, dpiv, &ar, s))) return e;
    if ((e = mat_out(A, lda, dA, ldd, m, n, f32, s))) return e;
    CK(cudaMemcpyAsync(IPIV, dpiv, pbytes, cudaMemcpyDeviceToHost, s), "pivots out");
    const int info = lnb_status_read(c, s);
    if (info < 0) return info;
    /* the reference's convention: relative to the first row of each b-wide panel */
    for (int i = 0; i < mn; ++i) IPIV[i] -= (i / b) * b;
    return info;
}

int ompss_dgetrf(int m, int n, int b, double *A, int lda, int *IPIV) { return getrf_host(m, n, b, A, lda, IPIV, 0); }
int ompss_sgetrf(int m, int n, int b, float *A, int lda, int *IPIV) { return getrf_host(m, n, b, A, lda, IPIV, 1); }
/* the left-looking drivers produce the same factorization (lull_main.c); on
 * the GPU both run the one schedule above */
int ompss_dgetrf_ll(int m, int n, int b, double *A, int lda, int *IPIV)
{
    return getrf_host(m, n, b, A, lda, IPIV, 0);
}
int ompss_sgetrf_ll(int m, int n, int b, float *A, int lda, int *IPIV)
{
    return getrf_host(m, n, b, A, lda, IPIV, 1);
}

static int gensolv_host(int m, int n, int b, void *A, void *B, int single)
{
    if (m < 0 || n < 0 || b <= 0) return lnb_set_error(LNB_EINVAL, "gensolv arguments m=%d n=%d b=%d", m, n, b);
    if (m == 0) return 0;
    if (!A || (n > 0 && !B)) return lnb_set_error(LNB_EINVAL, "gensolv: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ld_dev(m);
    const size_t abytes = (size_t)ldd * m * 8, bbytes = (size_t)ldd * (n ? n : 1) * 8, pbytes = (size_t)m * 4;
    const size_t fbytes = single ? (size_t)m * (m > n ? m : n) * 4 : 0;
    const size_t w1 = getrf_ws_bytes(m), w2 = lnb_trsm_f64_ws_bytes(m, n) + 1024;
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_align256(bbytes) + lnb_align256(pbytes) + lnb_align256(fbytes) +
                             (w1 > w2 ? w1 : w2));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, abytes), *dB = lnb_arena_take(&ar, bbytes);
    int *dpiv = lnb_arena_take(&ar, pbytes);
    float *f32 = single ? lnb_arena_take(&ar, fbytes) : NULL;
    cudaStream_t s = c->main;
    int e;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    if ((e = mat_in(dA, ldd, A, m, m, m, f32, s))) return e;
    if ((e = getrf_run(c, m, m, dA, ldd, dpiv, &ar, s))) return e;
    if ((e = mat_out(A, m, dA, ldd, m, m, f32, s))) return e;
    if (n > 0) {
        if ((e = mat_in(dB, ldd, B, m, m, n, f32, s))) return e;
        if ((e = getrs_run(c, m, n, dA, ldd, dpiv, dB, ldd, &ar, s))) return e;
        if ((e = mat_out(B, m, dB, ldd, m, n, f32, s))) return e;
    }
    return lnb_status_read(c, s);
}

int dgensolv_main(int m, int n, int b, double *A, double *B) { return gensolv_host(m, n, b, A, B, 0); }
int sgensolv_main(int m, int n, int b, float *A, float *B) { return gensolv_host(m, n, b, A, B, 1); }

/* ---- device-pointer entry points ---------------------------------------- */
int lnb_dgetrf_dev(int m, int n, double *dA, int lda, int *dipiv, int *info_dev, void *stream)
{
    if (m < 0 || n < 0 || lda < (m > 1 ? m : 1)) return lnb_set_error(LNB_EINVAL, "getrf sizes");
    if (m == 0 || n == 0) return 0;
    if (!dA || !dipiv) return lnb_set_error(LNB_EINVAL, "getrf: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, getrf_ws_bytes(n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    int e;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    if ((e = getrf_run(c, m, n, dA, lda, dipiv, &ar, s))) return e;
    if (info_dev) CK(cudaMemcpyAsync(info_dev, &c->st->info, sizeof(int), cudaMemcpyDeviceToDevice, s), "info");
    return 0;
}

int lnb_dgetrs_dev(int n, int nrhs, const double *dLU, int lda, const int *dipiv, double *dB, int ldb, void *stream)
{
    if (n < 0 || nrhs < 0 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "getrs sizes");
    if (n == 0 || nrhs == 0) return 0;
    if (!dLU || !dipiv || !dB) return lnb_set_error(LNB_EINVAL, "getrs: NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, lnb_trsm_f64_ws_bytes(n, nrhs) + 1024);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    return getrs_run(c, n, nrhs, dLU, lda, dipiv, dB, ldb, &ar, (cudaStream_t)stream);
}
