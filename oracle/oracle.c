/*
 * oracle.c -- CPU restatement of the Linompss tiled SPD-solve path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  The product library never links
 * or calls this file.  Pinned against outputs of the reference itself under
 * tests/golden/.
 *
 * Index arithmetic is 64-bit throughout: the reference's 32-bit `int`
 * offsets (e.g. chol_rlmain.c:27 `k*(lda+1)`) overflow above n = 46340.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((int64_t)(i) + (int64_t)(j) * (int64_t)(ld))

/* ------------------------------------------------------------------------ */
/* Tile operations (each one the semantics of one reference tile task).      */
/* The FP32 twins are generated from the same bodies.                        */
/* ------------------------------------------------------------------------ */

#define DEFINE_POTRF(NAME, T, SQRT)                                              \
int NAME(int64_t n, T *A, int64_t lda)                                           \
{                                                                                \
    /* Lower Cholesky, column by column (LAPACK xPOTF2 semantics).  On a       \
     * non-positive (or NaN) pivot the pivot is stored and info = j+1. */       \
    for (int64_t j = 0; j < n; ++j) {                                            \
        T d = A[IDX(j, j, lda)];                                                 \
        for (int64_t p = 0; p < j; ++p) d -= A[IDX(j, p, lda)] * A[IDX(j, p, lda)]; \
        if (!(d > (T)0)) { A[IDX(j, j, lda)] = d; return (int)(j + 1); }         \
        d = SQRT(d);                                                             \
        A[IDX(j, j, lda)] = d;                                                   \
        for (int64_t i = j + 1; i < n; ++i) {                                    \
            T s = A[IDX(i, j, lda)];                                             \
            for (int64_t p = 0; p < j; ++p) s -= A[IDX(i, p, lda)] * A[IDX(j, p, lda)]; \
            A[IDX(i, j, lda)] = s / d;                                           \
        }                                                                        \
    }                                                                            \
    return 0;                                                                    \
}

DEFINE_POTRF(orc_dpotrf, double, sqrt)
DEFINE_POTRF(orc_spotrf, float, sqrtf)

/* op(A)(i,j) for a triangular operand */
#define OPA(A, lda, trans, i, j) ((trans) == 'N' ? (A)[IDX(i, j, lda)] : (A)[IDX(j, i, lda)])

#define DEFINE_TRSM(NAME, T)                                                     \
void NAME(char side, char uplo, char trans, char diag, int64_t m, int64_t n,     \
          T alpha, const T *A, int64_t lda, T *B, int64_t ldb)                   \
{                                                                                \
    /* op(A) is lower when (uplo L, trans N) or (uplo U, trans T) */            \
    int oplower = (uplo == 'L') == (trans == 'N');                               \
    int unit = diag == 'U';                                                      \
    if (side == 'L') {                                                           \
        /* op(A) X = alpha B, A m x m */                                         \
        for (int64_t c = 0; c < n; ++c) {                                        \
            T *x = &B[IDX(0, c, ldb)];                                           \
            for (int64_t i = 0; i < m; ++i) x[i] *= alpha;                       \
            if (oplower) {                                                       \
                for (int64_t i = 0; i < m; ++i) {                                \
                    T s = x[i];                                                  \
                    for (int64_t p = 0; p < i; ++p) s -= OPA(A, lda, trans, i, p) * x[p]; \
                    x[i] = unit ? s : s / OPA(A, lda, trans, i, i);              \
                }                                                                \
            } else {                                                             \
                for (int64_t i = m - 1; i >= 0; --i) {                           \
                    T s = x[i];                                                  \
                    for (int64_t p = i + 1; p < m; ++p) s -= OPA(A, lda, trans, i, p) * x[p]; \
                    x[i] = unit ? s : s / OPA(A, lda, trans, i, i);              \
                }                                                                \
            }                                                                    \
        }                                                                        \
    } else {                                                                     \
        /* X op(A) = alpha B, A n x n; row r of X solves sum_p X(r,p) op(A)(p,j) */ \
        for (int64_t r = 0; r < m; ++r) {                                        \
            for (int64_t j = 0; j < n; ++j) B[IDX(r, j, ldb)] *= alpha;          \
            if (oplower) {                                                       \
                for (int64_t j = n - 1; j >= 0; --j) {                           \
                    T s = B[IDX(r, j, ldb)];                                     \
                    for (int64_t p = j + 1; p < n; ++p) s -= B[IDX(r, p, ldb)] * OPA(A, lda, trans, p, j); \
                    B[IDX(r, j, ldb)] = unit ? s : s / OPA(A, lda, trans, j, j); \
                }                                                                \
            } else {                                                             \
                for (int64_t j = 0; j < n; ++j) {                                \
                    T s = B[IDX(r, j, ldb)];                                     \
                    for (int64_t p = 0; p < j; ++p) s -= B[IDX(r, p, ldb)] * OPA(A, lda, trans, p, j); \
                    B[IDX(r, j, ldb)] = unit ? s : s / OPA(A, lda, trans, j, j); \
                }                                                                \
            }                                                                    \
        }                                                                        \
    }                                                                            \
}

DEFINE_TRSM(orc_dtrsm, double)
DEFINE_TRSM(orc_strsm, float)

#define DEFINE_SYRK(NAME, T)                                                     \
void NAME(char uplo, char trans, int64_t n, int64_t k, T alpha, const T *A,      \
          int64_t lda, T beta, T *C, int64_t ldc)                                \
{                                                                                \
    for (int64_t j = 0; j < n; ++j) {                                            \
        int64_t i0 = uplo == 'L' ? j : 0, i1 = uplo == 'L' ? n : j + 1;          \
        for (int64_t i = i0; i < i1; ++i) {                                      \
            T s = 0;                                                             \
            for (int64_t p = 0; p < k; ++p)                                      \
                s += trans == 'N' ? A[IDX(i, p, lda)] * A[IDX(j, p, lda)]        \
                                  : A[IDX(p, i, lda)] * A[IDX(p, j, lda)];       \
            C[IDX(i, j, ldc)] = (beta == (T)0 ? (T)0 : beta * C[IDX(i, j, ldc)]) + alpha * s; \
        }                                                                        \
    }                                                                            \
}

DEFINE_SYRK(orc_dsyrk, double)
DEFINE_SYRK(orc_ssyrk, float)

#define DEFINE_GEMM(NAME, T)                                                     \
void NAME(char transa, char transb, int64_t m, int64_t n, int64_t k, T alpha,    \
          const T *A, int64_t lda, const T *B, int64_t ldb, T beta, T *C,        \
          int64_t ldc)                                                           \
{                                                                                \
    for (int64_t j = 0; j < n; ++j)                                              \
        for (int64_t i = 0; i < m; ++i) {                                        \
            T s = 0;                                                             \
            for (int64_t p = 0; p < k; ++p) {                                    \
                T a = transa == 'N' ? A[IDX(i, p, lda)] : A[IDX(p, i, lda)];     \
                T b = transb == 'N' ? B[IDX(p, j, ldb)] : B[IDX(j, p, ldb)];     \
                s += a * b;                                                      \
            }                                                                    \
            C[IDX(i, j, ldc)] = (beta == (T)0 ? (T)0 : beta * C[IDX(i, j, ldc)]) + alpha * s; \
        }                                                                        \
}

DEFINE_GEMM(orc_dgemm, double)
DEFINE_GEMM(orc_sgemm, float)

static inline int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* Tile Cholesky drivers                                                      */
/* ------------------------------------------------------------------------ */

/* Right-looking, column-major (chol_rlmain.c:22-53).  Step k factors the
 * diagonal tile, solves the panel below it, then updates every trailing tile:
 * GEMM for (i,j) with j<i, SYRK for (i,i).  Two reference quirks are not
 * reproduced: the panel TRSM row count at chol_rlmain.c:36 uses the relative
 * row offset (it writes up to b-1 extra rows into the unused upper triangle
 * when n % b != 0), and chol_rlmain.c:45,48 index with n instead of lda.
 * Neither changes the lower triangle when lda == n. */
#define DEFINE_CHOL_RL(NAME, T, POTRF, TRSM, SYRK, GEMM)                         \
int NAME(int64_t n, int64_t b, T *A, int64_t lda)                                \
{                                                                                \
    int info = 0;                                                                \
    for (int64_t k = 0; k < n; k += b) {                                         \
        int64_t bs = min64(b, n - k);                                            \
        int ti = POTRF(bs, &A[IDX(k, k, lda)], lda);                             \
        if (ti && !info) info = (int)(k + ti);                                   \
        for (int64_t i = k + b; i < n; i += b)                                   \
            TRSM('R', 'L', 'T', 'N', min64(b, n - i), bs, (T)1,                  \
                 &A[IDX(k, k, lda)], lda, &A[IDX(i, k, lda)], lda);              \
        for (int64_t i = k + b; i < n; i += b) {                                 \
            int64_t ibs = min64(b, n - i);                                       \
            for (int64_t j = k + b; j < i; j += b)                               \
                GEMM('N', 'T', ibs, b, bs, (T)-1, &A[IDX(i, k, lda)], lda,       \
                     &A[IDX(j, k, lda)], lda, (T)1, &A[IDX(i, j, lda)], lda);    \
            SYRK('L', 'N', ibs, bs, (T)-1, &A[IDX(i, k, lda)], lda, (T)1,        \
                 &A[IDX(i, i, lda)], lda);                                       \
        }                                                                        \
    }                                                                            \
    return info;                                                                 \
}

DEFINE_CHOL_RL(orc_dchol_rl, double, orc_dpotrf, orc_dtrsm, orc_dsyrk, orc_dgemm)
DEFINE_CHOL_RL(orc_schol_rl, float, orc_spotrf, orc_strsm, orc_ssyrk, orc_sgemm)

/* Left-looking, column-major (chol_llmain.c:23-57): step k first applies all
 * previous panels to the diagonal tile (SYRK) and to the tiles below it
 * (GEMM), then factors the diagonal tile and solves the column below it. */
int orc_dchol_ll(int64_t n, int64_t b, double *A, int64_t lda)
{
    int info = 0;
    for (int64_t k = 0; k < n; k += b) {
        int64_t bs = min64(b, n - k);
        for (int64_t j = 0; j < k; j += b)
            orc_dsyrk('L', 'N', bs, b, -1.0, &A[IDX(k, j, lda)], lda, 1.0, &A[IDX(k, k, lda)], lda);
        int ti = orc_dpotrf(bs, &A[IDX(k, k, lda)], lda);
        if (ti && !info) info = (int)(k + ti);
        for (int64_t i = k + b; i < n; i += b) {
            int64_t ibs = min64(b, n - i);
            for (int64_t j = 0; j < k; j += b)
                orc_dgemm('N', 'T', ibs, b, b, -1.0, &A[IDX(i, j, lda)], lda,
                          &A[IDX(k, j, lda)], lda, 1.0, &A[IDX(i, k, lda)], lda);
            orc_dtrsm('R', 'L', 'T', 'N', ibs, b, 1.0, &A[IDX(k, k, lda)], lda,
                      &A[IDX(i, k, lda)], lda);
        }
    }
    return info;
}

/* Hypermatrix right-looking (chol_hrlmain.c:16-37): Ah[j*mt+i] is tile (i,j). */
int orc_dchol_hrl(int64_t mt, int64_t b, double **Ah)
{
    int info = 0;
    for (int64_t k = 0; k < mt; ++k) {
        int ti = orc_dpotrf(b, Ah[k * mt + k], b);
        if (ti && !info) info = (int)(k * b + ti);
        for (int64_t i = k + 1; i < mt; ++i)
            orc_dtrsm('R', 'L', 'T', 'N', b, b, 1.0, Ah[k * mt + k], b, Ah[k * mt + i], b);
        for (int64_t i = k + 1; i < mt; ++i) {
            for (int64_t j = k + 1; j < i; ++j)
                orc_dgemm('N', 'T', b, b, b, -1.0, Ah[k * mt + i], b, Ah[k * mt + j], b,
                          1.0, Ah[j * mt + i], b);
            orc_dsyrk('L', 'N', b, b, -1.0, Ah[k * mt + i], b, 1.0, Ah[i * mt + i], b);
        }
    }
    return info;
}

/* Hypermatrix left-looking (chol_hllmain.c:17-45). */
int orc_dchol_hll(int64_t mt, int64_t b, double **Ah)
{
    int info = 0;
    for (int64_t k = 0; k < mt; ++k) {
        for (int64_t j = 0; j < k; ++j)
            orc_dsyrk('L', 'N', b, b, -1.0, Ah[j * mt + k], b, 1.0, Ah[k * mt + k], b);
        int ti = orc_dpotrf(b, Ah[k * mt + k], b);
        if (ti && !info) info = (int)(k * b + ti);
        for (int64_t i = k + 1; i < mt; ++i) {
            for (int64_t j = 0; j < k; ++j)
                orc_dgemm('N', 'T', b, b, b, -1.0, Ah[j * mt + i], b, Ah[j * mt + k], b,
                          1.0, Ah[k * mt + i], b);
            orc_dtrsm('R', 'L', 'T', 'N', b, b, 1.0, Ah[k * mt + k], b, Ah[k * mt + i], b);
        }
    }
    return info;
}

/* ------------------------------------------------------------------------ */
/* Blocked left triangular solve (bblas_trsm.h:116-202)                       */
/* ------------------------------------------------------------------------ */
void orc_dltrsm(char uplo, char trans, char diag, int64_t bm, int64_t m, int64_t n,
                double alpha, const double *A, int64_t lda, double *B, int64_t ldb)
{
    if (uplo == 'L' && trans == 'N') {
        /* top-down: B_i = alpha B_i - sum_{j<i} A_ij X_j, then X_i = A_ii^-1 B_i */
        orc_dtrsm('L', 'L', 'N', diag, min64(bm, m), n, alpha, A, lda, B, ldb);
        for (int64_t i = bm; i < m; i += bm) {
            int64_t dimA = min64(bm, m - i);
            orc_dgemm('N', 'N', dimA, n, bm, -1.0, &A[IDX(i, 0, lda)], lda, &B[IDX(0, 0, ldb)], ldb,
                      alpha, &B[IDX(i, 0, ldb)], ldb);
            for (int64_t j = bm; j < i; j += bm)
                orc_dgemm('N', 'N', dimA, n, bm, -1.0, &A[IDX(i, j, lda)], lda, &B[IDX(j, 0, ldb)], ldb,
                          1.0, &B[IDX(i, 0, ldb)], ldb);
            orc_dtrsm('L', 'L', 'N', diag, dimA, n, 1.0, &A[IDX(i, i, lda)], lda, &B[IDX(i, 0, ldb)], ldb);
        }
    } else if (uplo == 'L') {
        /* lower, transposed: bottom-up; the last (ragged) block first */
        int64_t bR = m % bm > 0 ? m % bm : bm;
        int64_t boffs = m - bR;
        orc_dtrsm('L', 'L', 'T', diag, bR, n, alpha, &A[IDX(boffs, boffs, lda)], lda, &B[IDX(boffs, 0, ldb)], ldb);
        int64_t step = bm;
        for (int64_t j = boffs - bm; j >= 0; j -= bm, step += bm) {
            orc_dgemm('T', 'N', bm, n, bR, -1.0, &A[IDX(boffs, j, lda)], lda, &B[IDX(boffs, 0, ldb)], ldb,
                      alpha, &B[IDX(j, 0, ldb)], ldb);
            for (int64_t i = bm; i < step; i += bm)
                orc_dgemm('T', 'N', bm, n, bm, -1.0, &A[IDX(boffs - i, j, lda)], lda,
                          &B[IDX(boffs - i, 0, ldb)], ldb, 1.0, &B[IDX(j, 0, ldb)], ldb);
            orc_dtrsm('L', 'L', 'T', diag, bm, n, 1.0, &A[IDX(j, j, lda)], lda, &B[IDX(j, 0, ldb)], ldb);
        }
    } else if (trans == 'N') {
        /* upper, not transposed: bottom-up */
        int64_t bR = m % bm > 0 ? m % bm : bm;
        int64_t boffs = m - bR;
        orc_dtrsm('L', 'U', 'N', diag, bR, n, alpha, &A[IDX(boffs, boffs, lda)], lda, &B[IDX(boffs, 0, ldb)], ldb);
        int64_t step = bm;
        for (int64_t i = boffs - bm; i >= 0; i -= bm, step += bm) {
            orc_dgemm('N', 'N', bm, n, bR, -1.0, &A[IDX(i, boffs, lda)], lda, &B[IDX(boffs, 0, ldb)], ldb,
                      alpha, &B[IDX(i, 0, ldb)], ldb);
            for (int64_t j = bm; j < step; j += bm)
                orc_dgemm('N', 'N', bm, n, bm, -1.0, &A[IDX(i, boffs - j, lda)], lda,
                          &B[IDX(boffs - j, 0, ldb)], ldb, 1.0, &B[IDX(i, 0, ldb)], ldb);
            orc_dtrsm('L', 'U', 'N', diag, bm, n, 1.0, &A[IDX(i, i, lda)], lda, &B[IDX(i, 0, ldb)], ldb);
        }
    } else {
        /* upper, transposed: top-down */
        orc_dtrsm('L', 'U', 'T', diag, min64(bm, m), n, alpha, A, lda, B, ldb);
        for (int64_t j = bm; j < m; j += bm) {
            int64_t dimA = min64(bm, m - j);
            orc_dgemm('T', 'N', dimA, n, bm, -1.0, &A[IDX(0, j, lda)], lda, &B[IDX(0, 0, ldb)], ldb,
                      alpha, &B[IDX(j, 0, ldb)], ldb);
            for (int64_t i = bm; i < j; i += bm)
                orc_dgemm('T', 'N', dimA, n, bm, -1.0, &A[IDX(i, j, lda)], lda, &B[IDX(i, 0, ldb)], ldb,
                          1.0, &B[IDX(j, 0, ldb)], ldb);
            orc_dtrsm('L', 'U', 'T', diag, dimA, n, 1.0, &A[IDX(j, j, lda)], lda, &B[IDX(j, 0, ldb)], ldb);
        }
    }
}

/* dspdsolv_main (spdsolv_main.c:10-20) */
int orc_dspdsolv(int64_t m, int64_t nrhs, int64_t b, double *A, double *B)
{
    int info = orc_dchol_rl(m, b, A, m);
    orc_dltrsm('L', 'N', 'N', b, m, nrhs, 1.0, A, m, B, m);
    orc_dltrsm('L', 'T', 'N', b, m, nrhs, 1.0, A, m, B, m);
    return info;
}

/* ------------------------------------------------------------------------ */
/* Tile LU with partial pivoting (lu_main.c:5-27, lu_kernels.c:5-33) and the  */
/* general solve (gensolv_main.c:10-25)                                      */
/* ------------------------------------------------------------------------ */

/* TASK_GETRF (lu_kernels.c:5-10) is LAPACK dgetrf on the (m-j) x dimC panel,
 * restated unblocked (dgetf2): the pivot of column k is the first row of
 * largest |a| at or below k; rows k and p swap across the panel; the column
 * below the pivot is divided by it (skipped when it is exactly zero, which
 * sets info = k + 1); the rank-1 update follows.  ipiv is 1-based and
 * relative to the panel's first row, as dgetrf returns it for the panel. */
static int getf2(int64_t m, int64_t n, double *A, int64_t lda, int *ipiv)
{
    int info = 0;
    const int64_t mn = min64(m, n);
    for (int64_t k = 0; k < mn; ++k) {
        int64_t p = k;
        double amax = fabs(A[IDX(k, k, lda)]);
        for (int64_t i = k + 1; i < m; ++i) {
            const double v = fabs(A[IDX(i, k, lda)]);
            if (v > amax) { amax = v; p = i; }
        }
        ipiv[k] = (int)(p + 1);
        if (A[IDX(p, k, lda)] != 0.0) {
            if (p != k)
                for (int64_t j = 0; j < n; ++j) {
                    const double t = A[IDX(k, j, lda)];
                    A[IDX(k, j, lda)] = A[IDX(p, j, lda)];
                    A[IDX(p, j, lda)] = t;
                }
            for (int64_t i = k + 1; i < m; ++i) A[IDX(i, k, lda)] /= A[IDX(k, k, lda)];
        } else if (!info) {
            info = (int)(k + 1);
        }
        for (int64_t j = k + 1; j < n; ++j) {
            const double u = A[IDX(k, j, lda)];
            for (int64_t i = k + 1; i < m; ++i) A[IDX(i, j, lda)] -= A[IDX(i, k, lda)] * u;
        }
    }
    return info;
}

/* LAPACK dlaswp on ncols columns: rows k and ipiv[k]-1 swap for k = k1..k2-1 */
static void laswp(int64_t ncols, double *A, int64_t lda, int64_t k1, int64_t k2, const int *ipiv)
{
    for (int64_t k = k1; k < k2; ++k) {
        const int64_t p = ipiv[k] - 1;
        if (p == k) continue;
        for (int64_t j = 0; j < ncols; ++j) {
            const double t = A[IDX(k, j, lda)];
            A[IDX(k, j, lda)] = A[IDX(p, j, lda)];
            A[IDX(p, j, lda)] = t;
        }
    }
}

/* dlu_main (lu_main.c:5-27), m >= n: for each panel j of width dimC, getrf on
 * rows j..m-1; its swaps applied to dimC columns of every block column on the
 * left (TASK_LASWP: the reference passes the panel's width as the column
 * count, so with a ragged last panel the earlier blocks' columns past dimC are
 * not swapped); each block column on the right takes the swaps, a unit-lower
 * TRSM with the panel's top block and a GEMM with the rest of the panel
 * (TASK_TRSM_GEMM, lu_kernels.c:18-30).  ipiv[j..j+dimC) holds the panel's
 * pivots, 1-based and relative to row j.  Returns the first exactly zero
 * pivot's global column (1-based) or 0. */
int orc_dgetrf(int64_t m, int64_t n, int64_t b, double *A, int64_t lda, int *ipiv)
{
    int info = 0;
    for (int64_t j = 0; j < n; j += b) {
        const int64_t dimC = min64(b, n - j), dimR = m - j;
        if (dimR <= 0) break;
        int *ip = &ipiv[j];
        const int e = getf2(dimR, dimC, &A[IDX(j, j, lda)], lda, ip);
        if (e && !info) info = (int)(j + e);
        const int64_t ips = min64(dimR, dimC);
        for (int64_t jj = 0; jj < j; jj += b) laswp(dimC, &A[IDX(j, jj, lda)], lda, 0, ips, ip);
        for (int64_t jj = j + dimC; jj < n; jj += b) {
            const int64_t dimM = min64(b, n - jj);
            laswp(dimM, &A[IDX(j, jj, lda)], lda, 0, ips, ip);
            orc_dtrsm('L', 'L', 'N', 'U', dimC, dimM, 1.0, &A[IDX(j, j, lda)], lda, &A[IDX(j, jj, lda)], lda);
            orc_dgemm('N', 'N', dimR - dimC, dimM, dimC, -1.0, &A[IDX(j + dimC, j, lda)], lda, &A[IDX(j, jj, lda)],
                      lda, 1.0, &A[IDX(j + dimC, jj, lda)], lda);
        }
    }
    return info;
}

/* dgensolv_main (gensolv_main.c:10-25): A (m x m) = P L U by dlu_main; the
 * panels' swaps applied to B (m x n); then the blocked unit-lower and upper
 * solves.  As executed: the swap loop runs over i < n in steps of b and
 * applies panel i's pivots (relative to row i) starting at row b
 * (TASK_LASWP(b, ...)), which is where they belong only for i = b.  On the
 * reference's matrices (a +100 diagonal) no pivot leaves its row and the
 * swaps are all no-ops. */
int orc_dgensolv(int64_t m, int64_t n, int64_t b, double *A, double *B)
{
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)(m > n ? m : n));
    if (!ipiv) return -1;
    const int info = orc_dgetrf(m, m, b, A, m, ipiv);
    for (int64_t i = 0; i < n; i += b) {
        const int64_t dim = min64(b, n - i);
        laswp(n, &B[IDX(b, 0, m)], m, 0, dim, &ipiv[i]);
    }
    orc_dltrsm('L', 'N', 'U', b, m, n, 1.0, A, m, B, m);
    orc_dltrsm('U', 'N', 'N', b, m, n, 1.0, A, m, B, m);
    free(ipiv);
    return info;
}

/* ------------------------------------------------------------------------ */
/* Iterative refinement (itref.c)                                             */
/* ------------------------------------------------------------------------ */

/* y = alpha A x + beta y over bm-row blocks (bblas_dgemm as a matvec). */
static void matvec(int64_t n, const double *A, int64_t lda, const double *x, double alpha,
                   double beta, double *y)
{
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t p = 0; p < n; ++p) s += A[IDX(i, p, lda)] * x[p];
        y[i] = (beta == 0.0 ? 0.0 : beta * y[i]) + alpha * s;
    }
}

static double dot(int64_t n, int64_t bm, const double *x, const double *y)
{
    /* bblas_ddot: per-block partial sums added in block order (task_dot.c:30-59) */
    double total = 0.0;
    for (int64_t i = 0; i < n; i += bm) {
        int64_t c = min64(bm, n - i);
        double s = 0.0;
        for (int64_t p = 0; p < c; ++p) s += x[i + p] * y[i + p];
        total = (i == 0) ? s : total + s;
    }
    return total;
}

/* dcg_pure, dense, s = 1, not preconditioned, synchronous (itref.c:690-925).
 * The reference keeps every vector in buffer slot 0 (asman_nexti returns 0
 * and i never advances, itref.c:197,733,873), so the direction update of
 * itref.c:827, bblas_extm_daxpy(alpha1[i], alpha1[iprev], p[iprev], r[i],
 * p[i]), (1) reads the just-overwritten <r,r> through both pointers, so its
 * factor is exactly 1, and (2) runs task_axpy.c:89-97 with X and Z aliased:
 * Z = Y copies r into p first, then Z += f X adds the new p to itself.  The
 * effective recurrence is p = 2 r (a damped steepest descent after the
 * first step).  The restatement keeps that recurrence; it matches the
 * reference's iterates to rounding (tests/golden). */
int orc_dcg(int64_t n, int64_t bm, const double *A, int64_t lda, const double *b,
            double *x, double tol, int steps, double *res_log)
{
    double *r = malloc(sizeof(double) * n);
    double *p = malloc(sizeof(double) * n);
    double *tmp = malloc(sizeof(double) * n);
    double norm_b = sqrt(dot(n, n, b, b)); /* cblas_ddot over the whole vector */

    memcpy(r, b, sizeof(double) * n);
    matvec(n, A, lda, x, -1.0, 1.0, r);  /* r = b - A x */
    memcpy(p, r, sizeof(double) * n);
    double alpha1 = dot(n, bm, r, r);

    int converged = 0;
    int k;
    for (k = 0; k < steps; ++k) {
        matvec(n, A, lda, p, 1.0, 0.0, tmp);        /* tmp = A p */
        double alpha2 = dot(n, bm, tmp, p);         /* <tmp, p> */
        double f = alpha1 / alpha2;
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + f * p[i];
            r[i] = r[i] + (-1.0 * f) * tmp[i];
        }
        alpha1 = dot(n, bm, r, r);
        double beta = alpha1 / alpha1;              /* itref.c:827, see above */
        for (int64_t i = 0; i < n; ++i) {
            p[i] = r[i];                            /* Z = Y           */
            p[i] = p[i] + beta * p[i];              /* Z += f X, X == Z */
        }
        double sr2norm = sqrt(alpha1) / norm_b;
        if (res_log) res_log[k] = sr2norm;
        if (sr2norm <= tol) { converged = 1; break; }
    }
    free(r); free(p); free(tmp);
    return converged ? -1 : k;
}

/* Outer refinement loop of itref.c:999-1101, dense branch, refit > 0. */
int orc_ditref(int64_t n, int64_t bm, const double *A, const double *rhs, double *x,
               double prec, int refit, int it, double *norms)
{
    double *xs[2], *rs[2], *sd[2];
    double *buf = calloc((size_t)6 * n, sizeof(double));
    xs[0] = buf; xs[1] = buf + n; rs[0] = buf + 2 * n; rs[1] = buf + 3 * n;
    sd[0] = buf + 4 * n; sd[1] = buf + 5 * n;
    double r2norm[2] = {0.0, 0.0};

    /* initial solve from x = 0 */
    orc_dcg(n, bm, A, n, rhs, sd[1], prec, it, NULL);
    memcpy(xs[1], sd[1], sizeof(double) * n);
    memcpy(rs[1], rhs, sizeof(double) * n);
    matvec(n, A, n, xs[1], -1.0, 1.0, rs[1]);

    int prevb = 1;
    r2norm[1] = DBL_MAX;
    int i;
    for (i = 0; i < refit; ++i) {
        int b = i & 1;
        memset(sd[b], 0, sizeof(double) * n);
        orc_dcg(n, bm, A, n, rs[prevb], sd[b], prec, it, NULL);  /* A s = r */
        double sr2norm = sqrt(r2norm[prevb]);
        if (norms) norms[i] = sr2norm;
        if (sr2norm <= prec) { ++i; break; }
        for (int64_t q = 0; q < n; ++q) xs[b][q] = xs[prevb][q] + 1.0 * sd[b][q];
        memcpy(rs[b], rhs, sizeof(double) * n);
        matvec(n, A, n, xs[b], -1.0, 1.0, rs[b]);
        r2norm[b] = dot(n, bm, rs[b], rs[b]);
        prevb = b;
    }
    memcpy(x, xs[prevb], sizeof(double) * n);
    free(buf);
    return i;
}

/* ------------------------------------------------------------------------ */
/* Sparse refinement (itref.c built with USE_SPARSE)                           */
/* ------------------------------------------------------------------------ */
/* CSR matrices as hbmat_t holds them (hb.h:27-59): row pointers vptr[n+1],
 * column indices vpos and values vval, zero- or one-based (base = vptr[0],
 * the offset one2zero removes, itref_config.c:228-241). */

/* y = alpha A x + beta y.  The reference calls SBLAS_csrmv (bsblas_csrmm.h:
 * 214-232, one task per row block) which is MKL's mkl_dcsrmv with the
 * descriptor "GLNC" (general, zero-based): each row's products summed in
 * storage order, then scaled. */
void orc_csrmv(int64_t n, int base, const int *vptr, const int *vpos, const double *vval, const double *x,
               double alpha, double beta, double *y)
{
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t p = vptr[i] - base; p < vptr[i + 1] - base; ++p) s += vval[p] * x[vpos[p] - base];
        y[i] = (beta == 0.0 ? 0.0 : beta * y[i]) + alpha * s;
    }
}

/* Block-Jacobi preconditioner of itref_setup.c:55-93: the complete bm x bm
 * diagonal blocks of A (hb_sym_diag_block, hb.c:512-560), each factored by
 * Cholesky with natural ordering (cs_schol(A, 0) then cs_chol).  F holds
 * block k (order bk <= bm) dense at F + k bm bm, column-major with ld bm,
 * L in its lower part.  Returns 0, or 1 + the first block that is not
 * positive definite. */
int orc_bj_setup(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval, double *F)
{
    const int64_t nblk = (n + bm - 1) / bm;
    for (int64_t k = 0; k < nblk; ++k) {
        const int64_t r0 = k * bm, bk = min64(bm, n - r0);
        double *D = F + k * bm * bm;
        for (int64_t i = 0; i < bm * bm; ++i) D[i] = 0.0;
        for (int64_t r = r0; r < r0 + bk; ++r)
            for (int64_t p = vptr[r] - base; p < vptr[r + 1] - base; ++p) {
                const int64_t c = vpos[p] - base;
                if (c >= r0 && c < r0 + bk) D[(r - r0) + (c - r0) * bm] += vval[p];
            }
        for (int64_t j = 0; j < bk; ++j) {
            double d = D[j + j * bm];
            for (int64_t q = 0; q < j; ++q) d -= D[j + q * bm] * D[j + q * bm];
            if (!(d > 0.0)) return (int)(1 + k);
            d = sqrt(d);
            D[j + j * bm] = d;
            for (int64_t i = j + 1; i < bk; ++i) {
                double v = D[i + j * bm];
                for (int64_t q = 0; q < j; ++q) v -= D[i + q * bm] * D[j + q * bm];
                D[i + j * bm] = v / d;
            }
        }
    }
    return 0;
}

/* z = M^-1 r block by block: L L^T z_k = r_k (bsblas_dcholsolv2,
 * bsblas_csrmm.h:498-513, and cs_cholsol2 with the identity permutation) */
void orc_bj_apply(int64_t n, int64_t bm, const double *F, const double *r, double *z)
{
    const int64_t nblk = (n + bm - 1) / bm;
    for (int64_t k = 0; k < nblk; ++k) {
        const int64_t r0 = k * bm, bk = min64(bm, n - r0);
        const double *L = F + k * bm * bm;
        double *x = z + r0;
        for (int64_t i = 0; i < bk; ++i) x[i] = r[r0 + i];
        for (int64_t j = 0; j < bk; ++j) {           /* cs_lsolve: column-oriented */
            x[j] /= L[j + j * bm];
            for (int64_t i = j + 1; i < bk; ++i) x[i] -= L[i + j * bm] * x[j];
        }
        for (int64_t j = bk - 1; j >= 0; --j) {      /* cs_ltsolve */
            for (int64_t i = j + 1; i < bk; ++i) x[j] -= L[i + j * bm] * x[i];
            x[j] /= L[j + j * bm];
        }
    }
}

/* dcg_pure with the sparse matrix (itref.c:690-925, USE_SPARSE, s = 1,
 * synchronous branch), F = NULL for the unpreconditioned form.  The
 * recurrence as the reference executes it (every vector in slot 0, see
 * orc_dcg): with the preconditioner alpha1 = <r, z>, the direction update
 * is p = z then p += p (p = 2 z), and the relative test uses sqrt(alpha1). */
int orc_dscg(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval,
             const double *F, const double *b, double *x, double tol, int steps, double *res_log)
{
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n);
    double *tmp = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n);
    const double norm_b = sqrt(dot(n, n, b, b));
    memcpy(r, b, sizeof(double) * n);
    orc_csrmv(n, base, vptr, vpos, vval, x, -1.0, 1.0, r);     /* r = b - A x */
    double alpha1;
    if (F) {
        orc_bj_apply(n, bm, F, r, z);                            /* z = M^-1 r */
        memcpy(p, z, sizeof(double) * n);
        alpha1 = dot(n, bm, r, z);
    } else {
        memcpy(p, r, sizeof(double) * n);
        alpha1 = dot(n, bm, r, r);
    }
    int converged = 0, k;
    for (k = 0; k < steps; ++k) {
        orc_csrmv(n, base, vptr, vpos, vval, p, 1.0, 0.0, tmp);  /* tmp = A p (bsblas_dcg_comb) */
        const double alpha2 = dot(n, bm, p, tmp);
        const double f = alpha1 / alpha2;
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + f * p[i];
            r[i] = r[i] + (-1.0 * f) * tmp[i];
        }
        const double *y = r;
        if (F) {
            orc_bj_apply(n, bm, F, r, z);
            alpha1 = dot(n, bm, r, z);
            y = z;
        } else {
            alpha1 = dot(n, bm, r, r);
        }
        const double beta = alpha1 / alpha1;
        for (int64_t i = 0; i < n; ++i) {
            p[i] = y[i];
            p[i] = p[i] + beta * p[i];
        }
        const double sr2norm = sqrt(alpha1) / norm_b;
        if (res_log) res_log[k] = sr2norm;
        if (sr2norm <= tol) { converged = 1; break; }
    }
    free(r); free(p); free(tmp); free(z);
    return converged ? -1 : k;
}

/* The refinement loop of itref.c:999-1101 with the sparse matrix: the same
 * steps as orc_ditref, the residual by the CSR product. */
int orc_dsitref(int64_t n, int64_t bm, int base, const int *vptr, const int *vpos, const double *vval,
                const double *F, const double *rhs, double *x, double prec, int refit, int it, double *norms)
{
    double *xs[2], *rs[2], *sd[2];
    double *buf = calloc((size_t)6 * n, sizeof(double));
    xs[0] = buf; xs[1] = buf + n; rs[0] = buf + 2 * n; rs[1] = buf + 3 * n;
    sd[0] = buf + 4 * n; sd[1] = buf + 5 * n;
    double r2norm[2] = {0.0, DBL_MAX};
    orc_dscg(n, bm, base, vptr, vpos, vval, F, rhs, sd[1], prec, it, NULL);
    memcpy(xs[1], sd[1], sizeof(double) * n);
    memcpy(rs[1], rhs, sizeof(double) * n);
    orc_csrmv(n, base, vptr, vpos, vval, xs[1], -1.0, 1.0, rs[1]);
    int prevb = 1, i;
    for (i = 0; i < refit; ++i) {
        const int b = i & 1;
        memset(sd[b], 0, sizeof(double) * n);
        orc_dscg(n, bm, base, vptr, vpos, vval, F, rs[prevb], sd[b], prec, it, NULL);
        const double sr2norm = sqrt(r2norm[prevb]);
        if (norms) norms[i] = sr2norm;
        if (sr2norm <= prec) { ++i; break; }
        for (int64_t q = 0; q < n; ++q) xs[b][q] = xs[prevb][q] + 1.0 * sd[b][q];
        memcpy(rs[b], rhs, sizeof(double) * n);
        orc_csrmv(n, base, vptr, vpos, vval, xs[b], -1.0, 1.0, rs[b]);
        r2norm[b] = dot(n, bm, rs[b], rs[b]);
        prevb = b;
    }
    memcpy(x, xs[prevb], sizeof(double) * n);
    free(buf);
    return i;
}

/* ------------------------------------------------------------------------ */
/* Quality measures                                                           */
/* ------------------------------------------------------------------------ */
double orc_chol_residual(int64_t n, const double *A0, int64_t lda0, const double *L, int64_t ldl)
{
    /* || tril(L) tril(L)^T - A0 ||_inf / (||A0||_inf n eps)   (potrf_test.c:6-37) */
    double rnorm = 0.0, anorm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double rs = 0.0, as = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            int64_t kmax = i < j ? i : j;
            double s = 0.0;
            for (int64_t p = 0; p <= kmax; ++p) s += L[IDX(i, p, ldl)] * L[IDX(j, p, ldl)];
            rs += fabs(s - A0[IDX(i, j, lda0)]);
            as += fabs(A0[IDX(i, j, lda0)]);
        }
        if (rs > rnorm) rnorm = rs;
        if (as > anorm) anorm = as;
    }
    return rnorm / (anorm * (double)n * DBL_EPSILON / 2.0);
}

double orc_backward_error(int64_t n, int64_t nrhs, const double *A, int64_t lda,
                          const double *X, int64_t ldx, const double *B, int64_t ldb)
{
    double anorm = 0.0, xnorm = 0.0, bnorm = 0.0, rnorm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t j = 0; j < n; ++j) s += fabs(A[IDX(i, j, lda)]);
        if (s > anorm) anorm = s;
    }
    for (int64_t c = 0; c < nrhs; ++c)
        for (int64_t i = 0; i < n; ++i) {
            double r = B[IDX(i, c, ldb)];
            for (int64_t j = 0; j < n; ++j) r -= A[IDX(i, j, lda)] * X[IDX(j, c, ldx)];
            if (fabs(r) > rnorm) rnorm = fabs(r);
            if (fabs(X[IDX(i, c, ldx)]) > xnorm) xnorm = fabs(X[IDX(i, c, ldx)]);
            if (fabs(B[IDX(i, c, ldb)]) > bnorm) bnorm = fabs(B[IDX(i, c, ldb)]);
        }
    return rnorm / (anorm * xnorm + bnorm);
}
