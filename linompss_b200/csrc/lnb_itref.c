/*
 * lnb_itref.c -- the dense FP64 solver and refinement loop of itref.c (host C).
 *
 * ompss_dcg restates dcg_pure (itref.c:690-925, dense, s = 1, synchronous
 * branch) on device memory: r = b - A x, p = r, alpha1 = <r,r>; per step
 * tmp = A p, alpha2 = <tmp,p>, x += (alpha1/alpha2) p, r -= (alpha1/alpha2)
 * tmp, alpha1 = <r,r>, then the direction update as the reference executes
 * it (p = 2 r, see k_blas1.cu), and the relative test ||r||/||b|| <= tol.
 * The scalars never leave the device except the one norm per step that the
 * stopping test needs (the reference's taskwait, itref.c:830).
 *
 * ompss_ditref restates the outer loop of itref.c:999-1101.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

typedef struct {
    double *r, *p, *tmp;       /* n each */
    double *scal;              /* [0]=alpha1 [1]=alpha2 [2]=<b,b> [3]=spare */
    double *part, *dpart;
} cg_ws;

static size_t cg_ws_bytes(int64_t n)
{
    return 3 * lnb_align256((size_t)n * 8) + lnb_align256(8 * 8) +
           lnb_align256((size_t)lnb_gemv_part_doubles(n, n) * 8) +
           lnb_align256((size_t)lnb_dot_part_doubles(n) * 8) + 2048;
}

static int cg_ws_take(lnb_arena *ar, int64_t n, cg_ws *w)
{
    w->r = lnb_arena_take(ar, (size_t)n * 8);
    w->p = lnb_arena_take(ar, (size_t)n * 8);
    w->tmp = lnb_arena_take(ar, (size_t)n * 8);
    w->scal = lnb_arena_take(ar, 8 * 8);
    w->part = lnb_arena_take(ar, (size_t)lnb_gemv_part_doubles(n, n) * 8);
    w->dpart = lnb_arena_take(ar, (size_t)lnb_dot_part_doubles(n) * 8);
    return (w->r && w->p && w->tmp && w->scal && w->part && w->dpart) ? 0
                                                                       : lnb_set_error(LNB_ENOMEM, "cg workspace");
}

/* dcg_pure on device memory; mode 0 = the reference's recurrence.  Returns
 * -1 if converged, else the number of steps; < -1 (LNB_E*) on error. */
static int dcg_dev(lnb_ctx *c, int64_t n, const double *dA, int64_t lda, const double *db, double *dx,
                   double tol, int steps, int mode, cg_ws *w, cudaStream_t s)
{
    double *a1 = w->scal, *a2 = w->scal + 1, *bb = w->scal + 2;
    double h[2];
    CK(lnb_k_dot_f64(n, db, db, bb, w->dpart, s), "dot");
    /* r = b - A x;  p = r;  alpha1 = <r,r> */
    CK(lnb_k_gemv_f64(n, n, -1.0, dA, lda, dx, 1.0, db, w->r, w->r, a1, w->part, w->dpart, s), "gemv");
    CK(cudaMemcpyAsync(w->p, w->r, (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    CK(cudaMemcpyAsync(h, bb, 8, cudaMemcpyDeviceToHost, s), "read");
    CK(cudaStreamSynchronize(s), "sync");
    const double norm_b = sqrt(h[0]);
    int k;
    for (k = 0; k < steps; ++k) {
        /* tmp = A p, alpha2 = <tmp, p> */
        CK(lnb_k_gemv_f64(n, n, 1.0, dA, lda, w->p, 0.0, NULL, w->tmp, w->p, a2, w->part, w->dpart, s), "gemv");
        /* x += f p, r -= f tmp, alpha1 = <r,r> */
        CK(lnb_k_cg_xr_f64(n, a1, a2, w->p, w->tmp, dx, w->r, mode ? w->scal + 3 : a1, w->dpart, s), "cg xr");
        if (mode) {
            /* textbook: beta = new/old, then old <- new */
            CK(lnb_k_cg_p_f64(n, 1, w->scal + 3, a1, w->r, w->p, s), "cg p");
            CK(cudaMemcpyAsync(a1, w->scal + 3, 8, cudaMemcpyDeviceToDevice, s), "copy");
        } else {
            CK(lnb_k_cg_p_f64(n, 0, a1, a1, w->r, w->p, s), "cg p");
        }
        CK(cudaMemcpyAsync(h, a1, 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaStreamSynchronize(s), "sync");
        const double sr2norm = sqrt(h[0]) / norm_b;
        if (sr2norm <= tol) return -1;
    }
    return k;
}

static int copy_in_matrix(double *d, int64_t ldd, const double *h, int64_t ldh, int64_t n, cudaStream_t s)
{
    CK(cudaMemcpy2DAsync(d, (size_t)ldd * 8, h, (size_t)ldh * 8, (size_t)n * 8, (size_t)n,
                         cudaMemcpyHostToDevice, s), "A in");
    return 0;
}

int ompss_dcg(int n, int bm, const double *A, int lda, const double *b, double *x, double tol, int steps)
{
    (void)bm;
    if (n < 0 || lda < (n > 1 ? n : 1) || steps < 0) return lnb_set_error(LNB_EINVAL, "dcg arguments");
    if (n == 0) return -1;
    if (!A || !b || !x) return lnb_set_error(LNB_EINVAL, "NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = (n + 7) & ~7;
    void *ws = lnb_ws(c, lnb_align256((size_t)ldd * n * 8) + 2 * lnb_align256((size_t)n * 8) + cg_ws_bytes(n));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, (size_t)ldd * n * 8);
    double *db = lnb_arena_take(&ar, (size_t)n * 8), *dx = lnb_arena_take(&ar, (size_t)n * 8);
    cg_ws w;
    int e;
    if ((e = cg_ws_take(&ar, n, &w))) return e;
    cudaStream_t s = c->main;
    if ((e = copy_in_matrix(dA, ldd, A, lda, n, s))) return e;
    CK(cudaMemcpyAsync(db, b, (size_t)n * 8, cudaMemcpyHostToDevice, s), "b in");
    CK(cudaMemcpyAsync(dx, x, (size_t)n * 8, cudaMemcpyHostToDevice, s), "x in");
    int rc = dcg_dev(c, n, dA, ldd, db, dx, tol, steps, 0, &w, s);
    if (rc < -1) return rc;
    CK(cudaMemcpyAsync(x, dx, (size_t)n * 8, cudaMemcpyDeviceToHost, s), "x out");
    CK(cudaStreamSynchronize(s), "sync");
    return rc;
}

int ompss_ditref(int n, int bm, const double *A, int lda, const double *b, double *x, double prec,
                 int refit, int it, double *norms)
{
    (void)bm;
    if (n < 0 || lda < (n > 1 ? n : 1) || refit < 0 || it < 0) return lnb_set_error(LNB_EINVAL, "itref arguments");
    if (n == 0) return 0;
    if (!A || !b || !x) return lnb_set_error(LNB_EINVAL, "NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = (n + 7) & ~7;
    void *ws = lnb_ws(c, lnb_align256((size_t)ldd * n * 8) + 8 * lnb_align256((size_t)n * 8) + cg_ws_bytes(n) + 512);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, (size_t)ldd * n * 8);
    double *rhs = lnb_arena_take(&ar, (size_t)n * 8);
    double *xs[2], *rs[2], *sd[2];
    for (int i = 0; i < 2; ++i) {
        xs[i] = lnb_arena_take(&ar, (size_t)n * 8);
        rs[i] = lnb_arena_take(&ar, (size_t)n * 8);
        sd[i] = lnb_arena_take(&ar, (size_t)n * 8);
    }
    double *r2 = lnb_arena_take(&ar, 2 * 8);
    cg_ws w;
    int e;
    if ((e = cg_ws_take(&ar, n, &w))) return e;
    cudaStream_t s = c->main;
    if ((e = copy_in_matrix(dA, ldd, A, lda, n, s))) return e;
    CK(cudaMemcpyAsync(rhs, b, (size_t)n * 8, cudaMemcpyHostToDevice, s), "b in");
    CK(cudaMemsetAsync(sd[1], 0, (size_t)n * 8, s), "zero");
    /* initial solve from x = 0 (itref.c:1001-1006) */
    int rc = dcg_dev(c, n, dA, ldd, rhs, sd[1], prec, it, 0, &w, s);
    if (rc < -1) return rc;
    CK(cudaMemcpyAsync(xs[1], sd[1], (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    CK(lnb_k_gemv_f64(n, n, -1.0, dA, ldd, xs[1], 1.0, rhs, rs[1], NULL, NULL, w.part, w.dpart, s), "gemv");
    double r2norm[2] = {0.0, DBL_MAX};
    int prevb = 1, i;
    for (i = 0; i < refit; ++i) {
        const int bsel = i & 1;
        CK(cudaMemsetAsync(sd[bsel], 0, (size_t)n * 8, s), "zero");
        rc = dcg_dev(c, n, dA, ldd, rs[prevb], sd[bsel], prec, it, 0, &w, s);  /* A s = r */
        if (rc < -1) return rc;
        const double sr2norm = sqrt(r2norm[prevb]);
        if (norms) norms[i] = sr2norm;
        if (sr2norm <= prec) { ++i; break; }
        CK(lnb_k_axpy3_f64(n, 1.0, sd[bsel], xs[prevb], xs[bsel], s), "axpy");  /* x = x_prev + s */
        CK(lnb_k_gemv_f64(n, n, -1.0, dA, ldd, xs[bsel], 1.0, rhs, rs[bsel], rs[bsel], r2 + bsel, w.part,
                          w.dpart, s), "residual");                            /* r = b - A x, <r,r> */
        CK(cudaMemcpyAsync(&r2norm[bsel], r2 + bsel, 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaStreamSynchronize(s), "sync");
        prevb = bsel;
    }
    CK(cudaMemcpyAsync(x, xs[prevb], (size_t)n * 8, cudaMemcpyDeviceToHost, s), "x out");
    CK(cudaStreamSynchronize(s), "sync");
    return i;
}
