/*
 * lnb_mixed.c -- low-precision factor + FP64 iterative refinement (host C).
 *
 * The reference's refinement loop (itref.c:999-1101) keeps the residual
 * r = b - A x, the update x += s and the stopping test in FP64 and solves the
 * correction equation A s = r with an inner solver; its mixed-precision hooks
 * (bblas_d2s/s2d, itref.c:1009,1037) are commented out.  This driver makes
 * the low-precision path real:
 *
 *   1. As = S A S in FP32 (S = diag(1/sqrt(a_ii)) equilibration, optional),
 *      factored As = L L^T in FP32 storage with the trailing updates on the
 *      tensor cores (TF32x3 or per-block-scaled BF16) or SIMT FP32;
 *   2. refinement: z = S L^-T L^-1 S r (triangular solves read the FP32 factor
 *      and compute in FP64), x += z, r = b - A x in FP64 from the lower
 *      triangle of the untouched FP64 A, stop at the normwise backward error
 *      ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol (default 10 n eps);
 *   3. if refinement stalls (backward error not halving twice in a row, or
 *      growing), switch to CG preconditioned by the same factor, M^-1 =
 *      S L^-T L^-1 S, starting from the current x.
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

#define TRSV_H 64
#define LAPACK_EPS (DBL_EPSILON / 2.0)

int64_t lnb_trsm_blk_ints(int64_t n);
int64_t lnb_trsm_blk_inv_floats(int64_t n);
int64_t lnb_trsm_blk_vec_doubles(int64_t n, int64_t nrhs);
int lnb_trsm_blk_ok(const float *T, int64_t ldt, int64_t n, int64_t nrhs);
int lnb_k_trtri_hb_f32(const float *T, int64_t ldt, int64_t n, const float *dinv64, float *Binv, lnb_stream_t s);
int lnb_k_trsm_blk_f32(char trans, int64_t n, int64_t nrhs, const float *T, int64_t ldt, const float *Binv, double *B,
                       int64_t ldb, double *vec, int *sync, lnb_status_t *st, long long wait_ns, int sms,
                       lnb_stream_t s);
int lnb_k_coldot_f64(int64_t n, int64_t nrhs, const double *U, const double *V, double *out, lnb_stream_t s);
int lnb_k_pcg_xr_f64(int64_t n, int64_t nrhs, const double *num, const double *den, const double *P,
                     const double *Q, double *X, int64_t ldx, double *R, lnb_stream_t s);
int lnb_k_pcg_p_f64(int64_t n, int64_t nrhs, const double *num, const double *den, const double *Z, double *P,
                    lnb_stream_t s);

void lnb_ir_default_opts(lnb_ir_opts *o)
{
    if (!o) return;
    o->factor = LNB_FACTOR_TF32X3;
    o->max_iter = 30;
    o->tol = 0.0;
    o->equilibrate = 1;
    o->allow_pcg = 1;
    o->pcg_max_iter = 200;
}

typedef struct {
    int64_t n, nrhs, ld32;
    float *A32;
    double *S, *dinv, *R, *Z, *Y, *P, *Q, *scal; /* scal: 8 * nrhs scalars */
    double *rsum;           /* row sums of |A|, accumulated by the FP32 conversion */
    int *sync;
    /* solves on the inverses of the large diagonal blocks (k_trsv_blk.cu), when they apply */
    float *binv;
    double *bvec;
    int *bsync;
    int sms;
} irws;

static size_t ir_ws_bytes(int64_t n, int64_t nrhs, int b, int mode, int streamed)
{
    const int64_t ld32 = (n + 31) & ~(int64_t)31;
    const int64_t nb = (n + TRSV_H - 1) / TRSV_H;
    size_t s = lnb_align256((size_t)ld32 * n * 4) + lnb_align256((size_t)n * 8) * 2 +
               lnb_align256((size_t)nb * TRSV_H * TRSV_H * 8) + 5 * lnb_align256((size_t)n * nrhs * 8) +
               lnb_align256((size_t)8 * (nrhs + 1) * 8) +
               lnb_align256((size_t)lnb_trsm_sync_ints(n, TRSV_H) * 4) + 4096;
    s += lnb_align256((size_t)lnb_trsm_blk_inv_floats(n) * 4) +
         lnb_align256((size_t)lnb_trsm_blk_vec_doubles(n, nrhs) * 8) + lnb_align256((size_t)lnb_trsm_blk_ints(n) * 4);
    return s + (streamed ? lnb_chol_f32_stream_ws_bytes((int)n, b, mode) : lnb_chol_f32_ws_bytes((int)n, b, mode)) +
           lnb_refactor_ws_bytes(b);
}

/* z = M^-1 r = S L^-T L^-1 S r   (in place in Z, reading R) */
static int precond(lnb_ctx *c, const irws *w, cudaStream_t s)
{
    CK(lnb_k_scale_rows_f64(w->n, w->nrhs, w->S, w->R, w->Z, s), "scale");
    if (w->binv) {
        CK(lnb_k_trsm_blk_f32('N', w->n, w->nrhs, w->A32, w->ld32, w->binv, w->Z, w->n, w->bvec, w->bsync, c->st,
                              lnb_wait_ns(), w->sms, s), "forward solve");
        CK(lnb_k_trsm_blk_f32('T', w->n, w->nrhs, w->A32, w->ld32, w->binv, w->Z, w->n, w->bvec, w->bsync, c->st,
                              lnb_wait_ns(), w->sms, s), "backward solve");
        CK(lnb_k_scale_rows_f64(w->n, w->nrhs, w->S, w->Z, w->Z, s), "scale");
        return 0;
    }
    CK(lnb_k_trsm_left_f32('L', 'N', w->n, w->nrhs, 1.0, w->A32, w->ld32, (const float *)w->dinv, TRSV_H, w->Z, w->n, w->sync,
                           c->st, lnb_wait_ns(), 0, s), "forward solve");
    CK(lnb_k_trsm_left_f32('L', 'T', w->n, w->nrhs, 1.0, w->A32, w->ld32, (const float *)w->dinv, TRSV_H, w->Z, w->n, w->sync,
                           c->st, lnb_wait_ns(), 0, s), "backward solve");
    CK(lnb_k_scale_rows_f64(w->n, w->nrhs, w->S, w->Z, w->Z, s), "scale");
    return 0;
}

/* R = B - A X; returns the max over columns of the normwise backward error */
static int residual(lnb_ctx *c, const irws *w, const double *dA, int64_t lda, const double *dB, int64_t ldb,
                    const double *dX, int64_t ldx, double anorm, const double *bmax, double *be, cudaStream_t s)
{
    (void)c;
    const int64_t n = w->n, nrhs = w->nrhs;
    /* Q = X packed with ld n (Q is free here: PCG recomputes it each step), Y = A Q */
    CK(cudaMemcpy2DAsync(w->Q, n * 8, dX, ldx * 8, n * 8, nrhs, cudaMemcpyDeviceToDevice, s), "pack x");
    CK(lnb_k_symv_lower_f64(n, nrhs, dA, lda, w->Q, w->Y, 0, s), "symv");
    CK(lnb_k_resid_f64(n, nrhs, dB, ldb, w->Y, w->R, w->scal, s), "resid");
    CK(lnb_k_colmax_f64(n, nrhs, dX, ldx, w->scal + nrhs, s), "xmax");
    double h[2 * 64 + 2];
    const int64_t q2 = nrhs > 64 ? 64 : nrhs;
    CK(cudaMemcpyAsync(h, w->scal, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, s), "read");
    CK(cudaMemcpyAsync(h + 64, w->scal + nrhs, sizeof(double) * q2, cudaMemcpyDeviceToHost, s), "read");
    CK(cudaStreamSynchronize(s), "sync");
    double worst = 0.0;
    for (int64_t q = 0; q < q2; ++q) {
        const double den = anorm * h[64 + q] + bmax[q];
        const double e = den > 0 ? h[q] / den : 0.0;
        if (e > worst || e != e) worst = e;
    }
    *be = worst;
    return 0;
}

/* streamed input of the host entry point: A arrives block column by block
 * column (arr); the equilibration scale dS is already on the device */
typedef struct {
    const double *dS;
    cudaEvent_t *arr;
} ir_stream;

static int ir_run(lnb_ctx *c, int n, int nrhs, int b, const double *dA, int lda, const double *dB, int ldb,
                  double *dX, int ldx, const lnb_ir_opts *opts_in, lnb_ir_result *res, cudaStream_t s,
                  lnb_arena *arp, const ir_stream *in);

int lnb_dsposv_ir_dev(int n, int nrhs, int b, const double *dA, int lda, const double *dB, int ldb, double *dX,
                      int ldx, const lnb_ir_opts *opts_in, lnb_ir_result *res, void *stream)
{
    if (n < 0 || nrhs < 0 || b <= 0 || b > 1024 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) ||
        ldx < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "dsposv_ir arguments");
    if (nrhs > 64) return lnb_set_error(LNB_EINVAL, "dsposv_ir: nrhs = %d > 64", nrhs);
    const int mode = opts_in ? opts_in->factor : LNB_FACTOR_TF32X3;
    if (n == 0 || nrhs == 0) {
        if (res) memset(res, 0, sizeof *res);
        return 0;
    }
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    /* TF32 update paths with whole 32-blocks run the all-panels schedule (see
     * lnb_chol_f32_stream_run), which needs the larger workspace */
    void *ws = lnb_ws(c, ir_ws_bytes(n, nrhs, b, mode, lnb_chol_f32_stream_ok(n, b, mode)));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    return ir_run(c, n, nrhs, b, dA, lda, dB, ldb, dX, ldx, opts_in, res, (cudaStream_t)stream, &ar, NULL);
}

static int ir_run(lnb_ctx *c, int n, int nrhs, int b, const double *dA, int lda, const double *dB, int ldb,
                  double *dX, int ldx, const lnb_ir_opts *opts_in, lnb_ir_result *res, cudaStream_t s,
                  lnb_arena *arp, const ir_stream *in)
{
    lnb_ir_opts opts;
    if (opts_in) opts = *opts_in;
    else lnb_ir_default_opts(&opts);
    if (n < 0 || nrhs < 0 || b <= 0 || b > 1024 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) ||
        ldx < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "dsposv_ir arguments");
    if (nrhs > 64) return lnb_set_error(LNB_EINVAL, "dsposv_ir: nrhs = %d > 64", nrhs);
    int mode = opts.factor;
    if (mode != LNB_FACTOR_FP32 && mode != LNB_FACTOR_TF32X3 && mode != LNB_FACTOR_BF16 && mode != LNB_FACTOR_TF32)
        return lnb_set_error(LNB_EINVAL, "dsposv_ir: factor mode %d is not a low-precision mode", mode);
    lnb_ir_result rr;
    memset(&rr, 0, sizeof rr);
    if (n == 0 || nrhs == 0) { if (res) *res = rr; return 0; }
    lnb_arena ar = *arp;
    irws w;
    w.n = n; w.nrhs = nrhs; w.ld32 = ((int64_t)n + 31) & ~(int64_t)31;
    const int64_t nb = ((int64_t)n + TRSV_H - 1) / TRSV_H;
    w.A32 = lnb_arena_take(&ar, (size_t)w.ld32 * n * 4);
    w.S = lnb_arena_take(&ar, (size_t)n * 8);
    w.rsum = lnb_arena_take(&ar, (size_t)n * 8);
    w.dinv = lnb_arena_take(&ar, (size_t)nb * TRSV_H * TRSV_H * 8);
    w.R = lnb_arena_take(&ar, (size_t)n * nrhs * 8);
    w.Z = lnb_arena_take(&ar, (size_t)n * nrhs * 8);
    w.Y = lnb_arena_take(&ar, (size_t)n * nrhs * 8);
    w.P = lnb_arena_take(&ar, (size_t)n * nrhs * 8);
    w.Q = lnb_arena_take(&ar, (size_t)n * nrhs * 8);
    w.scal = lnb_arena_take(&ar, (size_t)8 * (nrhs + 1) * 8);
    w.sync = lnb_arena_take(&ar, (size_t)lnb_trsm_sync_ints(n, TRSV_H) * 4);
    if (!w.sync) return lnb_set_error(LNB_ENOMEM, "dsposv_ir workspace");
    w.sms = c->sms;
    w.binv = NULL;
    w.bvec = NULL;
    w.bsync = NULL;
    if (lnb_trsm_blk_ok(w.A32, w.ld32, n, nrhs)) {
        w.binv = lnb_arena_take(&ar, (size_t)lnb_trsm_blk_inv_floats(n) * 4);
        w.bvec = lnb_arena_take(&ar, (size_t)lnb_trsm_blk_vec_doubles(n, nrhs) * 8);
        w.bsync = lnb_arena_take(&ar, (size_t)lnb_trsm_blk_ints(n) * 4);
        if (!w.bsync) return lnb_set_error(LNB_ENOMEM, "dsposv_ir workspace");
    }
    const double tol = opts.tol > 0 ? opts.tol : 10.0 * n * LAPACK_EPS;

    /* ---- factor ---- */
    CK(cudaEventRecord(c->t0, s), "event");
    /* TF32 and FP32 factors: a first pass without per-step status reads (the
     * host queues the steps while the device runs them); a pivot that is not
     * positive shows in the final status, and the factor is then rebuilt from
     * the FP64 A on the checking path, which refactors that tile in FP64.
     * BF16 factors of ill-conditioned matrices fail often enough that the
     * rebuild would cost more than the per-step reads, so they check every
     * diagonal tile at once. */
    lnb_refactor_ctx rf = {dA, lda, w.S, 0, 0, mode == LNB_FACTOR_BF16};
    const lnb_arena ar_factor = ar;   /* a rerun carves the same workspace again */
    int e;
    /* the conversion to FP32 reads every element of the lower triangle once;
     * it also sums |A| by rows for ||A||_inf */
    CK(cudaMemsetAsync(w.rsum, 0, (size_t)n * 8, s), "row sums");
    /* on the streamed schedule the solves' diagonal-block inverses are formed
     * beside the factorization, as its diagonal tiles are finished */
    const lnb_blkinv inv = {(float *)w.dinv, w.binv};
    const int streamed = in || lnb_chol_f32_stream_ok(n, b, mode);
    if (in) {
        /* the matrix is converted block column by block column as it arrives */
        CK(cudaMemcpyAsync(w.S, in->dS, (size_t)n * 8, cudaMemcpyDeviceToDevice, s), "scale");
        const lnb_stream_in sin = {dA, lda, w.S, in->arr, w.rsum};
        e = lnb_chol_f32_stream_run(c, n, b, w.A32, w.ld32, mode, &rf, &sin, &inv, &ar, s);
    } else {
        CK(lnb_k_lower_to_f32(dA, lda, n, opts.equilibrate, w.S, w.A32, w.ld32, w.rsum, s), "convert");
        /* every panel's operands kept: columns beyond the look-ahead take their
         * panels two at a time, halving the passes over the trailing matrix */
        if (streamed)
            e = lnb_chol_f32_stream_run(c, n, b, w.A32, w.ld32, mode, &rf, NULL, &inv, &ar, s);
        else
            e = lnb_chol_f32_run(c, n, b, w.A32, w.ld32, mode, &rf, &ar, s);
    }
    if (!e && !rf.check) {
        const int info0 = lnb_status_read(c, s);
        if (info0 < 0) return info0;
        if (info0 > 0) {
            if (in) {
                /* every block column of A has landed before it is read again */
                const int nblk = (n + b - 1) / b;
                for (int j = 0; j < nblk; ++j) CK(cudaStreamWaitEvent(s, in->arr[j], 0), "arrival wait");
            }
            rf.check = 1;
            ar = ar_factor;
            CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
            /* the row sums are complete from the first pass */
            CK(lnb_k_lower_to_f32(dA, lda, n, opts.equilibrate, w.S, w.A32, w.ld32, NULL, s), "convert");
            if (streamed)
                e = lnb_chol_f32_stream_run(c, n, b, w.A32, w.ld32, mode, &rf, NULL, &inv, &ar, s);
            else
                e = lnb_chol_f32_run(c, n, b, w.A32, w.ld32, mode, &rf, &ar, s);
        }
    }
    rr.refactored_tiles = rf.refactored;
    if (e) {
        if (e > 0 && res) { rr.info = e; *res = rr; }
        return e > 0 ? lnb_set_error(e, "low-precision factor: tile at row %d could not be refactored", e) : e;
    }
    if (!streamed) {
        CK(lnb_k_trtri_blocks_f32(w.A32, w.ld32, n, TRSV_H, 'L', 0, (float *)w.dinv, s), "trtri");
        if (w.binv) CK(lnb_k_trtri_hb_f32(w.A32, w.ld32, n, (const float *)w.dinv, w.binv, s), "block inverses");
    }
    CK(cudaEventRecord(c->t1, s), "event");
    int info = lnb_status_read(c, s);
    if (info < 0) return info;
    rr.info = info;
    {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->t0, c->t1);
        rr.factor_ms = ms;
    }
    if (info > 0) {
        if (res) *res = rr;
        return lnb_set_error(info, "low-precision factor: leading minor %d not positive", info);
    }

    /* ---- norms ---- */
    CK(cudaEventRecord(c->t0, s), "event");
    double anorm, bmax[64];
    {
        /* ||A||_inf = max row sum of |A|, summed by the conversion */
        double h = 0.0;
        CK(lnb_k_colmax_f64(n, 1, w.rsum, n, w.scal, s), "max");
        CK(lnb_k_colmax_f64(n, nrhs, dB, ldb, w.scal + 1, s), "bmax");
        CK(cudaMemcpyAsync(&h, w.scal, 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaMemcpyAsync(bmax, w.scal + 1, (size_t)nrhs * 8, cudaMemcpyDeviceToHost, s), "read");
        CK(cudaStreamSynchronize(s), "sync");
        anorm = h;
    }

    /* ---- refinement ---- */
    CK(cudaMemset2DAsync(dX, (size_t)ldx * 8, 0, (size_t)n * 8, nrhs, s), "x = 0");
    CK(cudaMemcpy2DAsync(w.R, (size_t)n * 8, dB, (size_t)ldb * 8, (size_t)n * 8, nrhs, cudaMemcpyDeviceToDevice, s),
       "r = b");
    double be = INFINITY, be_prev = INFINITY;
    int slow = 0, it;
    for (it = 0; it < opts.max_iter; ++it) {
        if ((e = precond(c, &w, s))) return e;
        CK(lnb_k_axpy_scaled_f64(n, nrhs, NULL, w.Z, dX, ldx, s), "x += z");
        be_prev = be;
        if ((e = residual(c, &w, dA, lda, dB, ldb, dX, ldx, anorm, bmax, &be, s))) return e;
        if (be <= tol) { ++it; break; }
        if (!(be <= 0.5 * be_prev)) ++slow; else slow = 0;
        if (opts.allow_pcg && (slow >= 2 || be > be_prev)) { ++it; rr.used_pcg = 1; break; }
    }
    rr.iterations = it;

    /* ---- preconditioned CG fallback ---- */
    if (rr.used_pcg && be > tol) {
        double *rz = w.scal + 2 * (nrhs + 1), *pq = rz + nrhs + 1, *rz2 = pq + nrhs + 1;
        if ((e = precond(c, &w, s))) return e;                                 /* Z = M^-1 R */
        CK(cudaMemcpyAsync(w.P, w.Z, (size_t)n * nrhs * 8, cudaMemcpyDeviceToDevice, s), "p = z");
        CK(lnb_k_coldot_f64(n, nrhs, w.R, w.Z, rz, s), "rz");
        int k;
        for (k = 0; k < opts.pcg_max_iter; ++k) {
            CK(lnb_k_symv_lower_f64(n, nrhs, dA, lda, w.P, w.Q, 0, s), "Ap");
            CK(lnb_k_coldot_f64(n, nrhs, w.P, w.Q, pq, s), "pq");
            CK(lnb_k_pcg_xr_f64(n, nrhs, rz, pq, w.P, w.Q, dX, ldx, w.R, s), "x, r");
            if ((k & 3) == 3 || k + 1 == opts.pcg_max_iter) {
                /* true residual every 4 steps for the stopping test */
                if ((e = residual(c, &w, dA, lda, dB, ldb, dX, ldx, anorm, bmax, &be, s))) return e;
                if (be <= tol) { ++k; break; }
            }
            if ((e = precond(c, &w, s))) return e;
            CK(lnb_k_coldot_f64(n, nrhs, w.R, w.Z, rz2, s), "rz");
            CK(lnb_k_pcg_p_f64(n, nrhs, rz2, rz, w.Z, w.P, s), "p");
            CK(cudaMemcpyAsync(rz, rz2, (size_t)nrhs * 8, cudaMemcpyDeviceToDevice, s), "rz");
        }
        rr.pcg_iterations = k;
    }
    CK(cudaEventRecord(c->t1, s), "event");
    CK(cudaStreamSynchronize(s), "sync");
    {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->t0, c->t1);
        rr.solve_ms = ms;
    }
    {
        int st = lnb_status_read(c, s);
        if (st < 0) return st;
    }
    rr.backward_error = be;
    if (res) *res = rr;
    if (!(be <= tol))
        return lnb_set_error(LNB_ENOCONV, "refinement stopped at backward error %.3e > tol %.3e", be, tol);
    return 0;
}

int lnb_dsposv_ir(int n, int nrhs, int b, const double *A, int lda, const double *B, int ldb, double *X, int ldx,
                  const lnb_ir_opts *opts, lnb_ir_result *res)
{
    if (n < 0 || nrhs < 0 || b <= 0 || b > 1024 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1) ||
        ldx < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "dsposv_ir arguments");
    if (nrhs > 64) return lnb_set_error(LNB_EINVAL, "dsposv_ir: nrhs = %d > 64", nrhs);
    if (n == 0 || nrhs == 0) {
        if (res) memset(res, 0, sizeof *res);
        return 0;
    }
    if (!A || !B || !X) return lnb_set_error(LNB_EINVAL, "NULL argument");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int mode = opts ? opts->factor : LNB_FACTOR_TF32X3;
    /* the FP32 factorization starts while A is still crossing PCIe when the
     * mode allows it (TF32 update paths, b a multiple of 32) */
    const int streamed = lnb_chol_f32_stream_ok(n, b, mode);
    const int64_t ldd = ((int64_t)n + 7) & ~(int64_t)7;
    const size_t abytes = lnb_align256((size_t)ldd * n * 8), vbytes = lnb_align256((size_t)ldd * nrhs * 8);
    void *ws = lnb_ws(c, abytes + 2 * vbytes + lnb_align256((size_t)n * 8) + 1024 +
                          ir_ws_bytes(n, nrhs, b, mode, streamed));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = lnb_arena_take(&ar, (size_t)ldd * n * 8);
    double *dB = lnb_arena_take(&ar, (size_t)ldd * nrhs * 8);
    double *dX = lnb_arena_take(&ar, (size_t)ldd * nrhs * 8);
    double *dS = lnb_arena_take(&ar, (size_t)n * 8);
    if (!dS) return lnb_set_error(LNB_ENOMEM, "dsposv_ir: device buffers");
    cudaStream_t s = c->main;
    const int64_t cw = streamed ? b : 512;   /* block columns of the copy: the factor's tiles when streamed */
    const int nblk = (int)((n + cw - 1) / cw);
    double *diag = NULL;
    cudaEvent_t *arr = NULL;
    int e = 0, nev = 0;
    if (streamed) {
        diag = (double *)malloc((size_t)n * 8);
        arr = (cudaEvent_t *)calloc((size_t)nblk, sizeof(cudaEvent_t));
        if (!diag || !arr) e = lnb_set_error(LNB_ENOMEM, "host buffers");
        for (int64_t i = 0; !e && i < n; ++i) diag[i] = A[i + i * (int64_t)lda];
        for (; !e && nev < nblk; ++nev)
            if (cudaEventCreateWithFlags(&arr[nev], cudaEventDisableTiming) != cudaSuccess)
                e = lnb_cuda_error(cudaGetLastError(), "arrival events");
    }
    if (!e && cudaMemcpy2DAsync(dB, ldd * 8, B, (size_t)ldb * 8, (size_t)n * 8, nrhs, cudaMemcpyHostToDevice, s) !=
                  cudaSuccess)
        e = lnb_cuda_error(cudaGetLastError(), "B in");
    /* equilibration scale from the host-side diagonal, ahead of the bulk copy */
    if (!e && streamed) {
        if (cudaMemcpyAsync(dS, diag, (size_t)n * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)
            e = lnb_cuda_error(cudaGetLastError(), "diagonal");
        else if ((e = lnb_k_equil_scale_vec(dS, n, opts ? opts->equilibrate : 1, dS, s)) != 0)
            e = lnb_cuda_error(e, "scale");
    }
    /* lower block columns of A only (the solver never reads the upper
     * triangle); streamed, on the copy stream with an event per block column */
    cudaStream_t cs = streamed ? c->copy : s;
    for (int j = 0; j < nblk && !e; ++j) {
        const int64_t c0 = (int64_t)j * cw, wd = n - c0 < cw ? n - c0 : cw;
        if (cudaMemcpy2DAsync(dA + c0 + c0 * ldd, ldd * 8, A + c0 + c0 * (int64_t)lda, (size_t)lda * 8,
                              (size_t)(n - c0) * 8, wd, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
            (streamed && cudaEventRecord(arr[j], cs) != cudaSuccess))
            e = lnb_cuda_error(cudaGetLastError(), "A in");
    }
    if (!e) {
        const ir_stream in = {dS, arr};
        e = ir_run(c, n, nrhs, b, dA, (int)ldd, dB, (int)ldd, dX, (int)ldd, opts, res, s, &ar, streamed ? &in : NULL);
    }
    if (e >= 0 || e == LNB_ENOCONV) {
        if (cudaMemcpy2DAsync(X, (size_t)ldx * 8, dX, ldd * 8, (size_t)n * 8, nrhs, cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            e = lnb_cuda_error(cudaGetLastError(), "X out");
    }
    /* nothing may still be writing the cached buffers when this returns */
    if (streamed) cudaStreamSynchronize(c->copy);
    for (int j = 0; j < nev; ++j) cudaEventDestroy(arr[j]);
    free(arr);
    free(diag);
    return e;
}
