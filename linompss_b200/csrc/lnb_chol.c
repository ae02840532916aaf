/*
 * lnb_chol.c -- the right-looking tile Cholesky schedule (host C).
 *
 * Reference: dchol_rl (chol_rlmain.c:22-53) issues, for each k-step, one
 * POTRF task on the diagonal tile, one TRSM task per tile below it, and one
 * GEMM/SYRK task per trailing tile, which OmpSs runs as a DAG with POTRF/TRSM
 * at high priority (PRIOR_* chol_rlmain.c:16-19).
 *
 * Here each k-step is three launches: POTRF of the diagonal tile, one TRSM
 * over the whole panel below it, and the trailing SYRK+GEMM tasks fused into
 * lower-triangle DMMA updates.  The OmpSs priorities become a depth-2
 * look-ahead across two streams:
 *   crit (high priority): POTRF_k -> TRSM_k -> update of panel k+1 by panel k
 *   bulk (caller stream): update of panel k+2's columns, then the rest
 * so POTRF/TRSM of step k+1 run while the bulk update of step k streams
 * through the tensor cores.  ompss_dchol_ll / the hypermatrix forms produce
 * the same factor (the reference's variants differ only in task order), and
 * run this schedule too.
 */
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

/* one fused trailing-update launch (C[r,c] -= P[r,:] P[c,:], r >= c, c in
 * [c0,c1)), timed when diagnostics are on.  Algorithmic work: 2*k flops per
 * updated element; bytes: the panel rows read once per operand role plus
 * the updated elements read and written. */
static int upd(const double *P, int64_t ldp, double *C, int64_t ldc, int64_t nrows, int64_t c0,
               int64_t c1, int k, cudaStream_t s)
{
    const double w = (double)(c1 - c0);
    const double pairs = w * (double)nrows - (double)(c0 + c1 - 1) * w / 2.0;
    const int slot = lnb_prof_begin(s);
    int e = lnb_k_syrk_lower_f64(P, ldp, C, ldc, nrows, c0, c1, k, s);
    lnb_prof_end(slot, s, 2.0 * k * pairs,
                 8.0 * k * ((double)(nrows - c0) + w) + 16.0 * pairs);
    return e;
}

/* Factor the bs x bs diagonal tile at Akk on stream s.  Tiles up to 128 are
 * one leaf launch; larger tiles run a nested right-looking pass over 128-wide
 * sub-tiles (leaf POTRF, panel TRSM, DMMA update), the structure of the
 * reference's nested variant (chol_nrlmain.c).  Every leaf writes the
 * inverses of its own 32x32 diagonal blocks into dinv at its offset, so on
 * return dinv covers the whole tile. */
int lnb_potrf_tile_f64(double *Akk, int64_t lda, int bs, int64_t row0, double *dinv,
                          lnb_status_t *st, cudaStream_t s)
{
    const int LEAF_N = 128;
    for (int j = 0; j < bs; j += LEAF_N) {
        const int jb = bs - j < LEAF_N ? bs - j : LEAF_N;
        double *Ajj = Akk + j + (int64_t)j * lda;
        double *dj = dinv + (int64_t)(j / 32) * 1024;
        CK(lnb_k_potrf_f64(Ajj, lda, jb, row0 + j, dj, st, s), "potrf leaf");
        const int rem = bs - j - jb;
        if (rem > 0) {
            CK(lnb_k_trsm_rlt_f64(Ajj, lda, dj, Ajj + jb, lda, rem, jb, s), "potrf inner trsm");
            CK(lnb_k_syrk_lower_f64(Ajj + jb, lda, Ajj + jb + (int64_t)jb * lda, lda, rem, 0, rem, jb, s),
               "potrf inner update");
        }
    }
    return 0;
}

/* ---- schedule choice --------------------------------------------------------
 * LNB_SCHED_STREAMS: the host-issued two-stream look-ahead below (big fused
 * DMMA updates; best when the trailing matrix is large).
 * LNB_SCHED_DAG: one persistent launch that walks the tile DAG on the device
 * (k_chol_dag.cu; best when the critical path dominates).
 * LNB_SCHED_AUTO picks by size: the device DAG up to LNB_DAG_AUTO_MAX_N.
 * The environment variable LNB_CHOL_SCHED ("dag" / "streams") overrides the
 * process-wide setting. */
/* measured on B200 (b = 256 - 512): the DAG walk is ahead of the two-stream
 * schedule from n = 512 (0.37 vs 0.41 ms) to n = 16384 (53.1 vs 55.0 ms) */
#define LNB_DAG_AUTO_MAX_N 16384
static int g_sched = LNB_SCHED_AUTO;

void lnb_set_chol_schedule(int sched)
{
    if (sched == LNB_SCHED_AUTO || sched == LNB_SCHED_STREAMS || sched == LNB_SCHED_DAG) g_sched = sched;
}

int lnb_chol_f64_uses_dag(int n)
{
    const char *e = getenv("LNB_CHOL_SCHED");
    if (e && *e) {
        if (!strcmp(e, "dag")) return 1;
        if (!strcmp(e, "streams")) return 0;
    }
    if (g_sched == LNB_SCHED_DAG) return 1;
    if (g_sched == LNB_SCHED_STREAMS) return 0;
    return n <= LNB_DAG_AUTO_MAX_N;
}

size_t lnb_chol_f64_ws_bytes(int n, int b)
{
    return lnb_align256((size_t)((b + 31) / 32) * 1024 * sizeof(double)) + 256 +
           lnb_align256((size_t)lnb_chol_dag_w_doubles(n) * sizeof(double)) +
           lnb_align256((size_t)lnb_chol_dag_ints(n) * sizeof(int)) + 512;
}

/* the device-DAG schedule; w_out (may be NULL) receives the 64 x 64
 * diagonal-block inverses of L, the layout the triangular solves use */
static int chol_f64_dag(lnb_ctx *c, int n, double *dA, int64_t lda, lnb_arena *ar, cudaStream_t s,
                        double *copy_back, int64_t ldh, double **w_out)
{
    double *W = (double *)lnb_arena_take(ar, (size_t)lnb_chol_dag_w_doubles(n) * sizeof(double));
    int *sync = (int *)lnb_arena_take(ar, (size_t)lnb_chol_dag_ints(n) * sizeof(int));
    if (!W || !sync) return lnb_set_error(LNB_ENOMEM, "chol dag workspace");
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(lnb_k_chol_dag_f64(dA, lda, n, W, sync, c->st, lnb_wait_ns(), c->sms, 0, s), "chol dag");
    if (copy_back) {
        for (int64_t c0 = 0; c0 < n; c0 += 512) {
            const int64_t w = n - c0 < 512 ? n - c0 : 512;
            CK(cudaMemcpy2DAsync(copy_back + c0 + c0 * ldh, (size_t)ldh * sizeof(double), dA + c0 + c0 * lda,
                                 (size_t)lda * sizeof(double), (size_t)(n - c0) * sizeof(double), (size_t)w,
                                 cudaMemcpyDeviceToHost, s), "factor copy");
        }
    }
    if (w_out) *w_out = W;
    return 0;
}

int lnb_chol_f64_run_w(lnb_ctx *c, int n, int b, double *dA, int64_t lda, lnb_arena *ar, cudaStream_t s,
                       double *copy_back, int64_t ldh, double **w_out)
{
    if (w_out) *w_out = NULL;
    if (lnb_chol_f64_uses_dag(n)) return chol_f64_dag(c, n, dA, lda, ar, s, copy_back, ldh, w_out);
    return lnb_chol_f64_run(c, n, b, dA, lda, ar, s, copy_back, ldh);
}

int lnb_selftest_chol_wait_timeout(long long wait_us)
{
    /* 512 x 512 zeros.  The ticket starts at 1, so the first diagonal tile is
     * never factored and every task below it waits on a flag nothing sets. */
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t n = 512;
    void *ws = lnb_ws(c, lnb_align256(n * n * 8) + lnb_chol_f64_ws_bytes((int)n, 64));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *A = lnb_arena_take(&ar, n * n * 8);
    double *W = (double *)lnb_arena_take(&ar, (size_t)lnb_chol_dag_w_doubles(n) * sizeof(double));
    int *sync = (int *)lnb_arena_take(&ar, (size_t)lnb_chol_dag_ints(n) * sizeof(int));
    if (!sync) return lnb_set_error(LNB_ENOMEM, "self-test workspace");
    cudaStream_t s = c->main;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(cudaMemsetAsync(A, 0, n * n * 8, s), "zero");
    CK(lnb_k_chol_dag_f64(A, n, n, W, sync, c->st, (wait_us > 0 ? wait_us : 1000) * 1000LL, c->sms, 1, s),
       "chol dag");
    return lnb_status_read(c, s);
}

int lnb_chol_f64_run(lnb_ctx *c, int n, int b, double *dA, int64_t lda, lnb_arena *ar,
                     cudaStream_t s, double *copy_back, int64_t ldh)
{
    double *dinv = (double *)lnb_arena_take(ar, (size_t)((b + 31) / 32) * 1024 * sizeof(double));
    if (!dinv) return lnb_set_error(LNB_ENOMEM, "chol workspace");
    cudaStream_t crit = c->crit;
    cudaEvent_t ev_start = c->ev[0], ev_trsm = c->ev[1], ev_next = c->ev[2], ev_done = c->ev[3];

    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(cudaEventRecord(ev_start, s), "event");
    CK(cudaStreamWaitEvent(crit, ev_start, 0), "event wait");

    const int mt = (n + b - 1) / b;
    for (int k = 0; k < mt; ++k) {
        const int64_t k0 = (int64_t)k * b;
        const int bs = (int)(n - k0 < b ? n - k0 : b);
        double *Akk = dA + k0 + k0 * lda;
        const int64_t mrem = n - k0 - bs;      /* rows below the diagonal tile */

        /* panel factorization (crit) */
        { int _e = lnb_potrf_tile_f64(Akk, lda, bs, k0, dinv, c->st, crit); if (_e) return _e; }
        if (mrem > 0) CK(lnb_k_trsm_rlt_f64(Akk, lda, dinv, Akk + bs, lda, mrem, bs, crit), "trsm");
        CK(cudaEventRecord(ev_trsm, crit), "event");
        if (copy_back) {
            /* the panel is final: stream it back while later steps compute */
            CK(cudaStreamWaitEvent(c->copy, ev_trsm, 0), "event wait");
            CK(cudaMemcpy2DAsync(copy_back + k0 + k0 * ldh, (size_t)ldh * sizeof(double), Akk,
                                 (size_t)lda * sizeof(double), (size_t)(n - k0) * sizeof(double), bs,
                                 cudaMemcpyDeviceToHost, c->copy), "panel copy");
        }
        if (mrem <= 0) break;

        /* trailing update, origin at (k0+bs, k0+bs); P = panel rows below */
        const double *P = Akk + bs;
        double *Ct = Akk + bs + (int64_t)bs * lda;
        const int64_t nb1 = b < mrem ? b : mrem;               /* panel k+1 width */
        const int64_t nb2 = (2 * (int64_t)b) < mrem ? 2 * (int64_t)b : mrem;
        /* panel k+1 columns: on crit, right away */
        CK(upd(P, lda, Ct, lda, mrem, 0, nb1, bs, crit), "update next panel");
        /* the rest on the bulk stream once the panel is solved */
        CK(cudaStreamWaitEvent(s, ev_trsm, 0), "event wait");
        if (nb2 > nb1) {
            CK(upd(P, lda, Ct, lda, mrem, nb1, nb2, bs, s), "update panel k+2");
        }
        CK(cudaEventRecord(ev_next, s), "event");
        if (mrem > nb2) CK(upd(P, lda, Ct, lda, mrem, nb2, mrem, bs, s), "update rest");
        /* step k+1's own next-panel update needs panel k+2's columns current */
        CK(cudaStreamWaitEvent(crit, ev_next, 0), "event wait");
    }
    CK(cudaEventRecord(ev_done, crit), "event");
    CK(cudaStreamWaitEvent(s, ev_done, 0), "event wait");
    if (copy_back) {
        CK(cudaEventRecord(ev_done, c->copy), "event");
        CK(cudaStreamWaitEvent(s, ev_done, 0), "event wait");
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
static int check_args(int n, int b, const void *A, int lda)
{
    if (n < 0) return lnb_set_error(LNB_EINVAL, "n = %d < 0", n);
    if (b <= 0) return lnb_set_error(LNB_EINVAL, "tile size b = %d <= 0", b);
    if (lda < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "lda = %d < n = %d", lda, n);
    if (n > 0 && !A) return lnb_set_error(LNB_EINVAL, "A is NULL");
    if (b > 1024) return lnb_set_error(LNB_EINVAL, "tile size b = %d > 1024", b);
    return 0;
}

static inline int64_t ld_dev(int64_t n) { return (n + 7) & ~(int64_t)7; }

/* copy the lower block-columns (step columns each, rows from the block's
 * first column down) of a column-major matrix host<->device.  With step = b
 * every diagonal tile travels whole, which the panel copy-back relies on. */
static int copy_lower(double *dst, int64_t ldd, const double *src, int64_t lds, int64_t n,
                      int64_t step, enum cudaMemcpyKind kind, cudaStream_t s)
{
    for (int64_t c0 = 0; c0 < n; c0 += step) {
        int64_t w = n - c0 < step ? n - c0 : step;
        CK(cudaMemcpy2DAsync(dst + c0 + c0 * ldd, (size_t)ldd * sizeof(double), src + c0 + c0 * lds,
                             (size_t)lds * sizeof(double), (size_t)(n - c0) * sizeof(double), (size_t)w,
                             kind, s), "copy");
    }
    return 0;
}

static int chol_host(int n, int b, double *A, int lda)
{
    int e = check_args(n, b, A, lda);
    if (e) return e;
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ld_dev(n);
    const size_t abytes = (size_t)ldd * n * sizeof(double);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_chol_f64_ws_bytes(n, b));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = (double *)lnb_arena_take(&ar, abytes);
    cudaStream_t s = c->main;
    if ((e = copy_lower(dA, ldd, A, lda, n, b, cudaMemcpyHostToDevice, s))) return e;
    const int pinned = lnb_host_is_pinned(A);
    if ((e = lnb_chol_f64_run_w(c, n, b, dA, ldd, &ar, s, pinned ? A : NULL, lda, NULL))) return e;
    if (!pinned && (e = copy_lower(A, lda, dA, ldd, n, b, cudaMemcpyDeviceToHost, s))) return e;
    return lnb_status_read(c, s);
}

int ompss_dchol_rl(int n, int b, int t, double *A, int lda) { (void)t; return chol_host(n, b, A, lda); }
int ompss_dchol_ll(int n, int b, int t, double *A, int lda) { (void)t; return chol_host(n, b, A, lda); }

/* hypermatrix: gather tiles (i >= j) into a column-major device matrix */
static int chol_hyper(int mt, int b, double **Ah)
{
    if (mt < 0 || b <= 0 || b > 1024) return lnb_set_error(LNB_EINVAL, "mt = %d, b = %d", mt, b);
    if (mt == 0) return 0;
    if (!Ah) return lnb_set_error(LNB_EINVAL, "Ah is NULL");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t n = (int64_t)mt * b, ldd = ld_dev(n);
    const size_t abytes = (size_t)ldd * n * sizeof(double);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_chol_f64_ws_bytes((int)n, b));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    double *dA = (double *)lnb_arena_take(&ar, abytes);
    cudaStream_t s = c->main;
    for (int j = 0; j < mt; ++j)
        for (int i = j; i < mt; ++i) {
            const double *tile = Ah[(int64_t)j * mt + i];
            if (!tile) return lnb_set_error(LNB_EINVAL, "tile (%d,%d) is NULL", i, j);
            CK(cudaMemcpy2DAsync(dA + (int64_t)i * b + (int64_t)j * b * ldd, (size_t)ldd * sizeof(double),
                                 tile, (size_t)b * sizeof(double), (size_t)b * sizeof(double), (size_t)b,
                                 cudaMemcpyHostToDevice, s), "tile in");
        }
    int e = lnb_chol_f64_run_w(c, (int)n, b, dA, ldd, &ar, s, NULL, 0, NULL);
    if (e) return e;
    for (int j = 0; j < mt; ++j)
        for (int i = j; i < mt; ++i)
            CK(cudaMemcpy2DAsync(Ah[(int64_t)j * mt + i], (size_t)b * sizeof(double),
                                 dA + (int64_t)i * b + (int64_t)j * b * ldd, (size_t)ldd * sizeof(double),
                                 (size_t)b * sizeof(double), (size_t)b, cudaMemcpyDeviceToHost, s), "tile out");
    return lnb_status_read(c, s);
}

int ompss_dchol_hrl(int mt, int b, int t, double **Ah) { (void)t; return chol_hyper(mt, b, Ah); }
int ompss_dchol_hll(int mt, int b, int t, double **Ah) { (void)t; return chol_hyper(mt, b, Ah); }
int ompss_dchol_nhrl(int mt, int b, int t, double **Ah) { (void)t; return chol_hyper(mt, b, Ah); }
int ompss_dchol_nhll(int mt, int b, int t, double **Ah) { (void)t; return chol_hyper(mt, b, Ah); }

/* ---- device-pointer form ------------------------------------------------ */
int lnb_dchol_dev(int n, int b, double *dA, int lda, int *info_dev, void *stream)
{
    int e = check_args(n, b, dA, lda);
    if (e) return e;
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, lnb_chol_f64_ws_bytes(n, b));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    if ((e = lnb_chol_f64_run_w(c, n, b, dA, lda, &ar, s, NULL, 0, NULL))) return e;
    if (info_dev)
        CK(cudaMemcpyAsync(info_dev, &c->st->info, sizeof(int), cudaMemcpyDeviceToDevice, s), "info");
    return 0;
}
