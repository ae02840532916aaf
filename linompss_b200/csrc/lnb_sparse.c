/*
 * lnb_sparse.c -- the sparse FP64 refinement of itref.c built with USE_SPARSE
 * (host C), and a MatrixMarket reader for its input.
 *
 * ompss_dscg restates dcg_pure (itref.c:690-925) with the CSR matrix and,
 * when asked, the block-Jacobi preconditioner of itref_setup.c:55-93:
 *   r = b - A x; z = M^-1 r; p = z; alpha1 = <r, z>   (no preconditioner: z = r)
 *   per step: tmp = A p, alpha2 = <p, tmp> (bsblas_dcg_comb), x += f p,
 *   r -= f tmp with f = alpha1/alpha2; z = M^-1 r; alpha1 = <r, z>; then the
 *   direction update as the reference executes it (every vector in one slot,
 *   so p = z, p += p: p = 2 z), and the test sqrt(alpha1)/||b|| <= tol.
 * ompss_dsitref restates the outer loop of itref.c:999-1101 with the CSR
 * residual.  Device work: k_sparse.cu (CSR product, preconditioner) and
 * k_blas1.cu (deterministic dot products, the CG vector updates).
 */
#include <ctype.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

int lnb_k_csrmv_f64(int64_t n, int base, const int *vptr, const int *vpos, const double *vval, const double *x,
                    double alpha, double beta, const double *yin, double *y, lnb_stream_t s);
int64_t lnb_bj_doubles(int64_t n, int bm);
int64_t lnb_bj_env_ints(int64_t n, int bm);
int lnb_k_bj_setup(int64_t n, int bm, int base, const int *vptr, const int *vpos, const double *vval, double *fac,
                   int *env, int *info, lnb_stream_t s);
int lnb_k_bj_apply(int64_t n, int bm, const double *fac, const int *env, const double *r, double *z,
                   lnb_stream_t s);

#define BJ_MAX 512

typedef struct {
    int64_t n, nnz;
    int base, bm;
    int *vptr, *vpos;
    double *vval;
    double *fac;               /* block-Jacobi factors, NULL without the preconditioner */
    int *env;                  /* their envelopes per 32-row tile (the apply skips zero tiles) */
    double *r, *p, *tmp, *z;   /* n each */
    double *scal;              /* [0]=alpha1 [1]=alpha2 [2]=<b,b> [3]=<r,r> scratch */
    double *dpart;
} sp_ws;

static int check_csr(int n, const int *vptr, const int *vpos, const double *vval)
{
    if (n < 0) return lnb_set_error(LNB_EINVAL, "n = %d < 0", n);
    if (n == 0) return 0;
    if (!vptr || !vpos || !vval) return lnb_set_error(LNB_EINVAL, "NULL CSR array");
    const int base = vptr[0];
    if (base != 0 && base != 1) return lnb_set_error(LNB_EINVAL, "CSR base vptr[0] = %d (0 or 1)", base);
    for (int i = 0; i < n; ++i)
        if (vptr[i + 1] < vptr[i]) return lnb_set_error(LNB_EINVAL, "CSR row pointers decrease at row %d", i);
    const int64_t nnz = (int64_t)vptr[n] - base;
    for (int64_t p = 0; p < nnz; ++p)
        if (vpos[p] - base < 0 || vpos[p] - base >= n)
            return lnb_set_error(LNB_EINVAL, "CSR column index %d out of range at entry %lld", vpos[p], (long long)p);
    return 0;
}

static size_t sp_ws_bytes(int64_t n, int64_t nnz, int bm, int precond, int extra_vectors)
{
    size_t s = lnb_align256((size_t)(n + 1) * 4) + lnb_align256((size_t)nnz * 4) + lnb_align256((size_t)nnz * 8) +
               (4 + (size_t)extra_vectors) * lnb_align256((size_t)n * 8) + lnb_align256(8 * 8) +
               lnb_align256((size_t)lnb_dot_part_doubles(n) * 8) + 4096;
    if (precond)
        s += lnb_align256((size_t)lnb_bj_doubles(n, bm) * 8) + lnb_align256((size_t)((n + bm - 1) / bm) * 4) +
             lnb_align256((size_t)lnb_bj_env_ints(n, bm) * 4);
    return s;
}

/* upload the CSR matrix, build the preconditioner (bm <= 512) */
static int sp_setup(lnb_ctx *c, int n, int bm, const int *vptr, const int *vpos, const double *vval, int precond,
                    lnb_arena *ar, sp_ws *w, cudaStream_t s)
{
    w->n = n;
    w->base = vptr[0];
    w->nnz = (int64_t)vptr[n] - w->base;
    w->bm = bm;
    w->vptr = lnb_arena_take(ar, (size_t)(n + 1) * 4);
    w->vpos = lnb_arena_take(ar, (size_t)(w->nnz > 0 ? w->nnz : 1) * 4);
    w->vval = lnb_arena_take(ar, (size_t)(w->nnz > 0 ? w->nnz : 1) * 8);
    w->r = lnb_arena_take(ar, (size_t)n * 8);
    w->p = lnb_arena_take(ar, (size_t)n * 8);
    w->tmp = lnb_arena_take(ar, (size_t)n * 8);
    w->z = lnb_arena_take(ar, (size_t)n * 8);
    w->scal = lnb_arena_take(ar, 8 * 8);
    w->dpart = lnb_arena_take(ar, (size_t)lnb_dot_part_doubles(n) * 8);
    w->fac = NULL;
    if (!w->dpart) return lnb_set_error(LNB_ENOMEM, "sparse workspace");
    CK(cudaMemcpyAsync(w->vptr, vptr, (size_t)(n + 1) * 4, cudaMemcpyHostToDevice, s), "vptr in");
    if (w->nnz > 0) {
        CK(cudaMemcpyAsync(w->vpos, vpos, (size_t)w->nnz * 4, cudaMemcpyHostToDevice, s), "vpos in");
        CK(cudaMemcpyAsync(w->vval, vval, (size_t)w->nnz * 8, cudaMemcpyHostToDevice, s), "vval in");
    }
    if (precond) {
        const int nblk = (n + bm - 1) / bm;
        w->fac = lnb_arena_take(ar, (size_t)lnb_bj_doubles(n, bm) * 8);
        w->env = lnb_arena_take(ar, (size_t)lnb_bj_env_ints(n, bm) * 4);
        int *info = lnb_arena_take(ar, (size_t)nblk * 4);
        if (!info) return lnb_set_error(LNB_ENOMEM, "block-Jacobi workspace");
        CK(lnb_k_bj_setup(n, bm, w->base, w->vptr, w->vpos, w->vval, w->fac, w->env, info, s),
           "block-Jacobi factor");
        int *hinfo = (int *)malloc((size_t)nblk * 4);
        if (!hinfo) return lnb_set_error(LNB_ENOMEM, "host buffer");
        cudaError_t e = cudaMemcpyAsync(hinfo, info, (size_t)nblk * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        int bad = -1, piv = 0;
        for (int k = 0; e == cudaSuccess && k < nblk; ++k)
            if (hinfo[k] != 0) { bad = k; piv = hinfo[k]; break; }
        free(hinfo);
        if (e != cudaSuccess) return lnb_cuda_error(e, "block-Jacobi info");
        if (bad >= 0)
            return lnb_set_error(LNB_EINVAL, "block-Jacobi preconditioner: diagonal block %d (rows %d..) is not "
                                 "positive definite (pivot %d)", bad, bad * bm, piv);
    }
    (void)c;
    return 0;
}

/* z = M^-1 r (or a copy) */
static int sp_precond(const sp_ws *w, const double *r, double *z, cudaStream_t s)
{
    if (w->fac) CK(lnb_k_bj_apply(w->n, w->bm, w->fac, w->env, r, z, s), "block-Jacobi apply");
    else CK(cudaMemcpyAsync(z, r, (size_t)w->n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    return 0;
}

/* dcg_pure on device memory; returns -1 if converged, else the steps, < -1 on error */
static int dscg_dev(const sp_ws *w, const double *db, double *dx, double tol, int steps, cudaStream_t s)
{
    const int64_t n = w->n;
    double *a1 = w->scal, *a2 = w->scal + 1, *bb = w->scal + 2, *rr = w->scal + 3;
    double h = 0.0;
    CK(lnb_k_dot_f64(n, db, db, bb, w->dpart, s), "dot");
    /* r = b - A x;  z = M^-1 r;  p = z;  alpha1 = <r, z> */
    CK(lnb_k_csrmv_f64(n, w->base, w->vptr, w->vpos, w->vval, dx, -1.0, 1.0, db, w->r, s), "csrmv");
    int e;
    if ((e = sp_precond(w, w->r, w->z, s))) return e;
    CK(cudaMemcpyAsync(w->p, w->z, (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    CK(lnb_k_dot_f64(n, w->r, w->z, a1, w->dpart, s), "dot");
    CK(cudaMemcpyAsync(&h, bb, 8, cudaMemcpyDeviceToHost, s), "read");
    CK(cudaStreamSynchronize(s), "sync");
    const double norm_b = sqrt(h);
    int k;
    for (k = 0; k < steps; ++k) {
        CK(lnb_k_csrmv_f64(n, w->base, w->vptr, w->vpos, w->vval, w->p, 1.0, 0.0, NULL, w->tmp, s), "csrmv");
        CK(lnb_k_dot_f64(n, w->p, w->tmp, a2, w->dpart, s), "dot");
        CK(lnb_k_cg_xr_f64(n, a1, a2, w->p, w->tmp, dx, w->r, rr, w->dpart, s), "cg xr");
        if ((e = sp_precond(w, w->r, w->z, s))) return e;
        CK(lnb_k_dot_f64(n, w->r, w->z, a1, w->dpart, s), "dot");
        CK(lnb_k_cg_p_f64(n, 0, a1, a1, w->z, w->p, s), "cg p");        /* p = 2 z */
        CK(cudaMemcpyAsync(&h, a1, 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaStreamSynchronize(s), "sync");
        if (sqrt(h) / norm_b <= tol) return -1;
    }
    return k;
}

static int sp_args(int n, int bm, const int *vptr, const int *vpos, const double *vval, int precond)
{
    int e = check_csr(n, vptr, vpos, vval);
    if (e) return e;
    if (precond && (bm < 1 || bm > BJ_MAX))
        return lnb_set_error(LNB_EINVAL, "block-Jacobi block order bm = %d outside 1..%d", bm, BJ_MAX);
    if (!precond && bm < 1) return lnb_set_error(LNB_EINVAL, "bm = %d < 1", bm);
    return 0;
}

int ompss_dscg(int n, int bm, const int *vptr, const int *vpos, const double *vval, const double *b, double *x,
               double tol, int steps, int is_precond)
{
    int e = sp_args(n, bm, vptr, vpos, vval, is_precond);
    if (e) return e;
    if (steps < 0) return lnb_set_error(LNB_EINVAL, "steps = %d < 0", steps);
    if (n == 0) return -1;
    if (!b || !x) return lnb_set_error(LNB_EINVAL, "NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t nnz = (int64_t)vptr[n] - vptr[0];
    void *ws = lnb_ws(c, sp_ws_bytes(n, nnz, bm, is_precond, 2));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = c->main;
    sp_ws w;
    if ((e = sp_setup(c, n, bm, vptr, vpos, vval, is_precond, &ar, &w, s))) return e;
    double *db = lnb_arena_take(&ar, (size_t)n * 8), *dx = lnb_arena_take(&ar, (size_t)n * 8);
    if (!dx) return lnb_set_error(LNB_ENOMEM, "sparse workspace");
    CK(cudaMemcpyAsync(db, b, (size_t)n * 8, cudaMemcpyHostToDevice, s), "b in");
    CK(cudaMemcpyAsync(dx, x, (size_t)n * 8, cudaMemcpyHostToDevice, s), "x in");
    const int rc = dscg_dev(&w, db, dx, tol, steps, s);
    if (rc < -1) return rc;
    CK(cudaMemcpyAsync(x, dx, (size_t)n * 8, cudaMemcpyDeviceToHost, s), "x out");
    CK(cudaStreamSynchronize(s), "sync");
    return rc;
}

int ompss_dsitref(int n, int bm, const int *vptr, const int *vpos, const double *vval, const double *b, double *x,
                  double prec, int refit, int it, int is_precond, double *norms)
{
    int e = sp_args(n, bm, vptr, vpos, vval, is_precond);
    if (e) return e;
    if (refit < 0 || it < 0) return lnb_set_error(LNB_EINVAL, "sitref arguments");
    if (n == 0) return 0;
    if (!b || !x) return lnb_set_error(LNB_EINVAL, "NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t nnz = (int64_t)vptr[n] - vptr[0];
    void *ws = lnb_ws(c, sp_ws_bytes(n, nnz, bm, is_precond, 8));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = c->main;
    sp_ws w;
    if ((e = sp_setup(c, n, bm, vptr, vpos, vval, is_precond, &ar, &w, s))) return e;
    double *rhs = lnb_arena_take(&ar, (size_t)n * 8);
    double *xs[2], *rs[2], *sd[2];
    for (int i = 0; i < 2; ++i) {
        xs[i] = lnb_arena_take(&ar, (size_t)n * 8);
        rs[i] = lnb_arena_take(&ar, (size_t)n * 8);
        sd[i] = lnb_arena_take(&ar, (size_t)n * 8);
    }
    double *r2 = lnb_arena_take(&ar, 2 * 8);
    if (!r2) return lnb_set_error(LNB_ENOMEM, "sparse workspace");
    CK(cudaMemcpyAsync(rhs, b, (size_t)n * 8, cudaMemcpyHostToDevice, s), "b in");
    CK(cudaMemsetAsync(sd[1], 0, (size_t)n * 8, s), "zero");
    /* initial solve from x = 0 (itref.c:1000-1006), r = b - A x (itref.c:1013-1015) */
    int rc = dscg_dev(&w, rhs, sd[1], prec, it, s);
    if (rc < -1) return rc;
    CK(cudaMemcpyAsync(xs[1], sd[1], (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "copy");
    CK(lnb_k_csrmv_f64(n, w.base, w.vptr, w.vpos, w.vval, xs[1], -1.0, 1.0, rhs, rs[1], s), "residual");
    double r2norm[2] = {0.0, DBL_MAX};
    int prevb = 1, i;
    for (i = 0; i < refit; ++i) {
        const int bsel = i & 1;
        CK(cudaMemsetAsync(sd[bsel], 0, (size_t)n * 8, s), "zero");
        rc = dscg_dev(&w, rs[prevb], sd[bsel], prec, it, s);                   /* A s = r */
        if (rc < -1) return rc;
        const double sr2norm = sqrt(r2norm[prevb]);
        if (norms) norms[i] = sr2norm;
        if (sr2norm <= prec) { ++i; break; }
        CK(lnb_k_axpy3_f64(n, 1.0, sd[bsel], xs[prevb], xs[bsel], s), "axpy");   /* x = x_prev + s */
        CK(lnb_k_csrmv_f64(n, w.base, w.vptr, w.vpos, w.vval, xs[bsel], -1.0, 1.0, rhs, rs[bsel], s), "residual");
        CK(lnb_k_dot_f64(n, rs[bsel], rs[bsel], r2 + bsel, w.dpart, s), "dot");
        CK(cudaMemcpyAsync(&r2norm[bsel], r2 + bsel, 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaStreamSynchronize(s), "sync");
        prevb = bsel;
    }
    CK(cudaMemcpyAsync(x, xs[prevb], (size_t)n * 8, cudaMemcpyDeviceToHost, s), "x out");
    CK(cudaStreamSynchronize(s), "sync");
    return i;
}

/* ---- MatrixMarket coordinate files -> CSR ----------------------------------
 * The reference reads its sparse matrices from files (readHB_newmat_double,
 * itref_config.c:228-241) and expands a symmetric one stored as a triangle to
 * full storage (dhb_sym_expand).  This reader takes the MatrixMarket
 * coordinate form ("real" or "integer", "general" or "symmetric") and returns
 * zero-based CSR with every row's columns ascending; a symmetric file's
 * off-diagonal entries appear in both triangles. */
typedef struct { int r, c; double v; } mm_ent;

static int mm_cmp(const void *a, const void *b)
{
    const mm_ent *x = a, *y = b;
    if (x->r != y->r) return x->r < y->r ? -1 : 1;
    return (x->c > y->c) - (x->c < y->c);
}

int lnb_mm_read_csr(const char *path, int *n_out, int **vptr_out, int **vpos_out, double **vval_out)
{
    if (!path || !n_out || !vptr_out || !vpos_out || !vval_out) return lnb_set_error(LNB_EINVAL, "NULL argument");
    FILE *f = fopen(path, "r");
    if (!f) return lnb_set_error(LNB_EINVAL, "cannot open %s", path);
    char line[1024];
    int symmetric = 0, e = 0;
    if (!fgets(line, sizeof line, f)) { fclose(f); return lnb_set_error(LNB_EINVAL, "%s: empty file", path); }
    for (char *q = line; *q; ++q) *q = (char)tolower((unsigned char)*q);
    if (strncmp(line, "%%matrixmarket", 14) != 0 || !strstr(line, "matrix") || !strstr(line, "coordinate") ||
        !(strstr(line, "real") || strstr(line, "integer"))) {
        fclose(f);
        return lnb_set_error(LNB_EINVAL, "%s: not a real/integer MatrixMarket coordinate file", path);
    }
    if (strstr(line, "symmetric")) symmetric = 1;
    else if (!strstr(line, "general")) {
        fclose(f);
        return lnb_set_error(LNB_EINVAL, "%s: only general or symmetric storage", path);
    }
    long m = 0, nc = 0, nz = 0;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        if (sscanf(line, "%ld %ld %ld", &m, &nc, &nz) == 3) break;
    }
    if (m <= 0 || m != nc || nz < 0 || m > 2147483647L) {
        fclose(f);
        return lnb_set_error(LNB_EINVAL, "%s: a square matrix is required (%ld x %ld)", path, m, nc);
    }
    mm_ent *ent = malloc(sizeof(mm_ent) * (size_t)(symmetric ? 2 * nz : nz) + 1);
    if (!ent) { fclose(f); return lnb_set_error(LNB_ENOMEM, "host memory"); }
    long cnt = 0;
    for (long k = 0; k < nz && !e; ++k) {
        long i, j;
        double v;
        if (fscanf(f, "%ld %ld %lf", &i, &j, &v) != 3) e = lnb_set_error(LNB_EINVAL, "%s: entry %ld unreadable", path, k);
        else if (i < 1 || i > m || j < 1 || j > m) e = lnb_set_error(LNB_EINVAL, "%s: entry %ld out of range", path, k);
        else {
            ent[cnt++] = (mm_ent){(int)(i - 1), (int)(j - 1), v};
            if (symmetric && i != j) ent[cnt++] = (mm_ent){(int)(j - 1), (int)(i - 1), v};
        }
    }
    fclose(f);
    if (e) { free(ent); return e; }
    qsort(ent, (size_t)cnt, sizeof(mm_ent), mm_cmp);
    int *vptr = calloc((size_t)m + 1, sizeof(int));
    int *vpos = malloc(sizeof(int) * (size_t)(cnt ? cnt : 1));
    double *vval = malloc(sizeof(double) * (size_t)(cnt ? cnt : 1));
    if (!vptr || !vpos || !vval) {
        free(ent); free(vptr); free(vpos); free(vval);
        return lnb_set_error(LNB_ENOMEM, "host memory");
    }
    for (long k = 0; k < cnt; ++k) {
        vptr[ent[k].r + 1]++;
        vpos[k] = ent[k].c;
        vval[k] = ent[k].v;
    }
    for (long i = 0; i < m; ++i) vptr[i + 1] += vptr[i];
    free(ent);
    *n_out = (int)m;
    *vptr_out = vptr;
    *vpos_out = vpos;
    *vval_out = vval;
    return 0;
}

void lnb_mm_free(int *vptr, int *vpos, double *vval)
{
    free(vptr);
    free(vpos);
    free(vval);
}
