/*
 * lnb_chol32.c -- the FP32-storage tile Cholesky schedule (host C).
 *
 * Same right-looking schedule and depth-2 look-ahead as the FP64 one
 * (lnb_chol.c, after chol_rlmain.c:22-53), used for the FP32 twins
 * (ompss_schol_rl: schol_rl) and for the low-precision factor of the
 * mixed-precision solver.  The trailing update runs in one of three modes:
 *   LNB_FACTOR_FP32   SIMT FP32 (the plain single-precision tile tasks)
 *   LNB_FACTOR_TF32X3 tcgen05 kind::tf32, 3 products on the hi/lo split
 *   LNB_FACTOR_BF16   tcgen05 kind::f16, BF16 operands with per-block scales
 * For the tensor-core modes each solved panel is first rewritten as K-major
 * operand copies (k_prep_*), double-buffered across k-steps: the copy of
 * step k stays alive while the bulk update of step k runs, and step k+2's
 * copy only starts after that update (the crit stream waits on it).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

/* the triangular solves' diagonal blocks: 64 x 64 inverses, and 512 x 512 ones
 * built from them (k_trsv_blk.cu) */
#define TRSV_H 64
int lnb_k_trtri_hb_f32(const float *T, int64_t ldt, int64_t n, const float *dinv64, float *Binv, lnb_stream_t s);

static int g_schol_mode = LNB_FACTOR_TF32X3;

void lnb_set_factor_mode(int mode)
{
    if (mode == LNB_FACTOR_FP32 || mode == LNB_FACTOR_TF32X3 || mode == LNB_FACTOR_BF16 ||
        mode == LNB_FACTOR_TF32)
        g_schol_mode = mode;
}
int lnb_get_factor_mode(void) { return g_schol_mode; }

static inline int64_t kpad_of(int b) { return ((int64_t)b + 63) & ~(int64_t)63; }

size_t lnb_chol_f32_stream_ws_bytes(int n, int b, int mode);
int lnb_chol_f32_stream_ok(int n, int b, int mode);

size_t lnb_chol_f32_ws_bytes(int n, int b, int mode)
{
    /* TF32 paths with whole 32-blocks keep every panel's operands */
    if (lnb_chol_f32_stream_ok(n, b, mode)) return lnb_chol_f32_stream_ws_bytes(n, b, mode);
    size_t bytes = lnb_align256((size_t)((b + 31) / 32) * 1024 * sizeof(float)) + 256;
    const int64_t kp = kpad_of(b);
    if (mode == LNB_FACTOR_TF32X3) bytes += 4 * lnb_align256((size_t)n * kp * 4);
    else if (mode == LNB_FACTOR_TF32) bytes += 2 * lnb_align256((size_t)n * kp * 4);
    else if (mode == LNB_FACTOR_BF16)
        bytes += 2 * lnb_align256((size_t)n * kp * 2) + 2 * lnb_align256((size_t)(n / 128 + 2) * 4);
    return bytes + 4096;
}

/* one diagonal tile: a cluster launch (whole 32-blocks, up to 512), a leaf
 * (<= 128), or a nested 128-wide pass with SIMT inner updates; dinv receives
 * the tile's 32x32 block inverses */
int lnb_k_potrf_cluster_f32(float *A, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                            cudaStream_t s);

int lnb_potrf_tile_f32(float *Akk, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                       cudaStream_t s)
{
    const int LEAF_N = 128;
    /* whole 32-blocks, 16-byte aligned: one cluster launch */
    if (bs >= 64 && bs <= 512 && bs % 32 == 0 && (uintptr_t)Akk % 16 == 0 && lda % 4 == 0 &&
        (uintptr_t)dinv % 16 == 0) {
        CK(lnb_k_potrf_cluster_f32(Akk, lda, bs, row0, dinv, st, s), "potrf tile f32");
        return 0;
    }
    for (int j = 0; j < bs; j += LEAF_N) {
        const int jb = bs - j < LEAF_N ? bs - j : LEAF_N;
        float *Ajj = Akk + j + (int64_t)j * lda;
        float *dj = dinv + (int64_t)(j / 32) * 1024;
        CK(lnb_k_potrf_f32(Ajj, lda, jb, row0 + j, dj, st, s), "potrf leaf f32");
        const int rem = bs - j - jb;
        if (rem > 0) {
            CK(lnb_k_trsm_rlt_f32(Ajj, lda, dj, Ajj + jb, lda, rem, jb, s), "inner trsm f32");
            CK(lnb_k_syrk_lower_f32_simt(Ajj + jb, lda, Ajj + jb + (int64_t)jb * lda, lda, rem, 0, rem, jb, s),
               "inner update f32");
        }
    }
    return 0;
}

typedef struct {
    int mode;
    int64_t kpad;
    void *hi[2], *lo[2];
    float *scale[2];
} panelbuf;

int lnb_k_scaled_tile_f64(const double *A, int64_t lda, const double *s, int bs, double *T, int64_t ldt,
                          cudaStream_t st);
int lnb_k_f32_to_f64(const float *X, int64_t ldx, int64_t m, int64_t k, double *D, int64_t ldd, cudaStream_t st);
int lnb_k_f64_to_f32_lower(const double *T, int64_t ldt, int bs, float *X, int64_t ldx, cudaStream_t st);
int lnb_k_restore_shift(const double *src, double *T, int64_t ldt, int bs, double shift, cudaStream_t st);
int lnb_k_diag_absmax(const double *T, int64_t ldt, int bs, double *out, cudaStream_t st);
int lnb_k_dinv32_f32(const float *L, int64_t ldl, int bs, float *dinv, cudaStream_t st);

#define RF_KC 2048

size_t lnb_refactor_ws_bytes(int b)
{
    return 2 * lnb_align256((size_t)b * b * 8) + lnb_align256((size_t)b * RF_KC * 8) +
           lnb_align256((size_t)((b + 31) / 32) * 1024 * 8) + 1024;
}

/* FP64 diagonal-tile refactor after a failed low-precision pivot in tile
 * [k0, k0+bs): the tile's Schur complement is recomputed in FP64 from the
 * original matrix and the finished FP32 panel rows,
 *     T = S_k A_kk S_k - L_k,0:k0 L_k,0:k0^T,
 * factored in FP64 (with a growing diagonal shift if even that is not
 * positive definite), and written back as the FP32 factor tile together
 * with its 32x32 block inverses.  Returns 0 when the tile was repaired,
 * > 0 if it could not be. */
static int refactor_tile(lnb_ctx *c, lnb_refactor_ctx *rf, float *dA, int64_t lda, int64_t k0, int bs, int b,
                         float *dinv, lnb_arena *ar_in, cudaStream_t s)
{
    lnb_arena ar = *ar_in;   /* scratch is released on return */
    double *T = lnb_arena_take(&ar, (size_t)b * b * 8), *T0 = lnb_arena_take(&ar, (size_t)b * b * 8);
    double *chunk = lnb_arena_take(&ar, (size_t)b * RF_KC * 8);
    double *dinv64 = lnb_arena_take(&ar, (size_t)((b + 31) / 32) * 1024 * 8);
    if (!dinv64) return lnb_set_error(LNB_ENOMEM, "refactor workspace");
    CK(cudaMemsetAsync(&c->st->info, 0, sizeof(int), s), "info reset");
    CK(lnb_k_scaled_tile_f64(rf->A + k0 + k0 * rf->lda, rf->lda, rf->S + k0, bs, T, b, s), "tile");
    for (int64_t kc = 0; kc < k0; kc += RF_KC) {
        const int64_t kw = k0 - kc < RF_KC ? k0 - kc : RF_KC;
        CK(lnb_k_f32_to_f64(dA + k0 + kc * lda, lda, bs, kw, chunk, bs, s), "panel rows");
        CK(lnb_k_syrk_lower_f64(chunk, bs, T, b, bs, 0, bs, (int)kw, s), "schur");
    }
    CK(cudaMemcpyAsync(T0, T, (size_t)b * bs * 8, cudaMemcpyDeviceToDevice, s), "backup");
    double dmax = 0.0;
    int info = 1;
    for (int t = 0; t < 8 && info != 0; ++t) {
        if (t > 0) {
            if (t == 1) {
                CK(lnb_k_diag_absmax(T0, b, bs, chunk, s), "diag max");
                CK(cudaMemcpyAsync(&dmax, chunk, 8, cudaMemcpyDeviceToHost, s), "read");
                CK(cudaStreamSynchronize(s), "sync");
            }
            const double shift = dmax * ldexp(1.0, -24 + 4 * t);
            CK(lnb_k_restore_shift(T0, T, b, bs, shift, s), "shift");
            CK(cudaMemsetAsync(&c->st->info, 0, sizeof(int), s), "info reset");
            rf->shifted++;
        }
        { int e = lnb_potrf_tile_f64(T, b, bs, k0, dinv64, c->st, s); if (e) return e; }
        info = lnb_status_read(c, s);
        if (info < 0) return info;
    }
    if (info != 0) return info;
    CK(lnb_k_f64_to_f32_lower(T, b, bs, dA + k0 + k0 * lda, lda, s), "write back");
    CK(lnb_k_dinv32_f32(dA + k0 + k0 * lda, lda, bs, dinv, s), "block inverses");
    rf->refactored++;
    return 0;
}

static int upd32(const panelbuf *pb, int slot, const float *P, int64_t ldp, float *C, int64_t ldc,
                 int64_t nrows, int64_t c0, int64_t c1, int k, lnb_status_t *st, cudaStream_t s)
{
    const double w = (double)(c1 - c0);
    const double pairs = w * (double)nrows - (double)(c0 + c1 - 1) * w / 2.0;
    const int prof = lnb_prof_begin(s);
    int e;
    if (pb->mode == LNB_FACTOR_FP32) {
        e = lnb_k_syrk_lower_f32_simt(P, ldp, C, ldc, nrows, c0, c1, k, s);
    } else {
        const int m = pb->mode == LNB_FACTOR_TF32X3 ? 0 : pb->mode == LNB_FACTOR_TF32 ? 1 : 2;
        e = lnb_k_tc_syrk_lower(m, pb->hi[slot], pb->lo[slot], pb->kpad, nrows, C, ldc, nrows, c0, c1, k,
                                pb->scale[slot], st, lnb_wait_ns(), s);
    }
    const double opb = pb->mode == LNB_FACTOR_BF16 ? 2.0 : pb->mode == LNB_FACTOR_TF32X3 ? 8.0 : 4.0;
    lnb_prof_end(prof, s, 2.0 * k * pairs, opb * (double)pb->kpad * ((double)(nrows - c0) + w) + 8.0 * pairs);
    return e;
}

int lnb_chol_f32_run(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, lnb_refactor_ctx *rf,
                     lnb_arena *ar, cudaStream_t s)
{
    /* TF32 update paths with whole 32-blocks: every panel's operands kept, far
     * columns updated several panels at a time */
    if (lnb_chol_f32_stream_ok(n, b, mode))
        return lnb_chol_f32_stream_run(c, n, b, dA, lda, mode, rf, NULL, NULL, ar, s);
    float *dinv = (float *)lnb_arena_take(ar, (size_t)((b + 31) / 32) * 1024 * sizeof(float));
    if (!dinv) return lnb_set_error(LNB_ENOMEM, "chol32 workspace");
    panelbuf pb;
    memset(&pb, 0, sizeof pb);
    pb.mode = mode;
    pb.kpad = kpad_of(b);
    for (int i = 0; i < 2; ++i) {
        if (mode == LNB_FACTOR_TF32X3 || mode == LNB_FACTOR_TF32) {
            pb.hi[i] = lnb_arena_take(ar, (size_t)n * pb.kpad * 4);
            if (mode == LNB_FACTOR_TF32X3) pb.lo[i] = lnb_arena_take(ar, (size_t)n * pb.kpad * 4);
            if (!pb.hi[i] || (mode == LNB_FACTOR_TF32X3 && !pb.lo[i]))
                return lnb_set_error(LNB_ENOMEM, "panel copies");
        } else if (mode == LNB_FACTOR_BF16) {
            pb.hi[i] = lnb_arena_take(ar, (size_t)n * pb.kpad * 2);
            pb.scale[i] = (float *)lnb_arena_take(ar, (size_t)(n / 128 + 2) * 4);
            if (!pb.hi[i] || !pb.scale[i]) return lnb_set_error(LNB_ENOMEM, "panel copies");
        }
    }
    cudaStream_t crit = c->crit;
    cudaEvent_t ev_start = c->ev[0], ev_trsm = c->ev[1], ev_next = c->ev[2], ev_done = c->ev[3];
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    CK(cudaEventRecord(ev_start, s), "event");
    CK(cudaStreamWaitEvent(crit, ev_start, 0), "event wait");

    const int mt = (n + b - 1) / b;
    for (int k = 0; k < mt; ++k) {
        const int64_t k0 = (int64_t)k * b;
        const int bs = (int)(n - k0 < b ? n - k0 : b);
        float *Akk = dA + k0 + k0 * lda;
        const int64_t mrem = n - k0 - bs;
        const int slot = k & 1;
        { int _e = lnb_potrf_tile_f32(Akk, lda, bs, k0, dinv, c->st, crit); if (_e) return _e; }
        if (rf && rf->check) {
            /* the refinement driver wants a usable factor: check this tile now */
            int info = lnb_status_read(c, crit);
            if (info < 0) return info;
            if (info > 0) {
                int e = refactor_tile(c, rf, dA, lda, k0, bs, b, dinv, ar, crit);
                if (e) return e;
            }
        }
        if (mrem > 0) {
            if (mode == LNB_FACTOR_TF32X3 || mode == LNB_FACTOR_TF32) {
                /* panel solve with the K-major operand copies written by the same launch */
                CK(lnb_k_trsm_rlt_prep_f32(Akk, lda, dinv, Akk + bs, lda, mrem, bs, (float *)pb.hi[slot],
                                           mode == LNB_FACTOR_TF32X3 ? (float *)pb.lo[slot] : NULL, (int)pb.kpad,
                                           crit), "trsm+prep f32");
            } else {
                CK(lnb_k_trsm_rlt_f32(Akk, lda, dinv, Akk + bs, lda, mrem, bs, crit), "trsm f32");
                if (mode == LNB_FACTOR_BF16)
                    CK(lnb_k_prep_bf16(Akk + bs, lda, mrem, bs, (int)pb.kpad, pb.scale[slot], pb.hi[slot], crit),
                       "prep bf16");
            }
        }
        CK(cudaEventRecord(ev_trsm, crit), "event");
        if (mrem <= 0) break;
        const float *P = Akk + bs;
        float *Ct = Akk + bs + (int64_t)bs * lda;
        const int64_t nb1 = b < mrem ? b : mrem;
        const int64_t nb2 = (2 * (int64_t)b) < mrem ? 2 * (int64_t)b : mrem;
        CK(upd32(&pb, slot, P, lda, Ct, lda, mrem, 0, nb1, bs, c->st, crit), "update next panel");
        CK(cudaStreamWaitEvent(s, ev_trsm, 0), "event wait");
        if (nb2 > nb1) CK(upd32(&pb, slot, P, lda, Ct, lda, mrem, nb1, nb2, bs, c->st, s), "update panel k+2");
        CK(cudaEventRecord(ev_next, s), "event");
        if (mrem > nb2) CK(upd32(&pb, slot, P, lda, Ct, lda, mrem, nb2, mrem, bs, c->st, s), "update rest");
        CK(cudaStreamWaitEvent(crit, ev_next, 0), "event wait");
    }
    CK(cudaEventRecord(ev_done, crit), "event");
    CK(cudaStreamWaitEvent(s, ev_done, 0), "event wait");
    return 0;
}

/* ---- streamed input ----------------------------------------------------------
 * The matrix arrives over PCIe block column by block column while the
 * factorization runs.  The K-major operand copies of every panel are kept (one
 * n x ldk array each for hi and lo; panel k fills K columns [k b, k b + b) of
 * the rows below it), so a block column that arrives after some panels are
 * done is brought up to date by one long-K update with all of them (a
 * left-looking "catch-up") and from then on takes the right-looking updates.
 * A column joins as soon as its data is there -- the host checks the arrival
 * events every step, and the per-step status read keeps it within a step of
 * the device -- and at the latest when the next panels need it, in which case
 * the device waits for its arrival event. */

static inline int64_t ldk_of(int n) { return ((int64_t)n + 31) & ~(int64_t)31; }

/* LNB_STREAM_AHEAD caps how many block columns beyond the next two may join
 * early (unset: no cap); 0 makes every column join by a catch-up update just
 * before it is needed */
static int stream_ahead(void)
{
    const char *e = getenv("LNB_STREAM_AHEAD");
    return (e && *e) ? atoi(e) : 1 << 30;
}

int lnb_chol_f32_stream_ok(int n, int b, int mode)
{
    return (mode == LNB_FACTOR_TF32X3 || mode == LNB_FACTOR_TF32) && b % 32 == 0 && n > b;
}

size_t lnb_chol_f32_stream_ws_bytes(int n, int b, int mode)
{
    size_t bytes = lnb_align256((size_t)((b + 31) / 32) * 1024 * sizeof(float)) + 256;
    bytes += (mode == LNB_FACTOR_TF32X3 ? 2 : 1) * lnb_align256((size_t)n * ldk_of(n) * 4);
    return bytes + 4096;
}

static int upd_tc(int mode, const float *hi, const float *lo, int64_t kstride, float *C, int64_t ldc, int64_t nrows,
                  int64_t c0, int64_t c1, int k, lnb_status_t *st, cudaStream_t s)
{
    if (nrows <= c0 || c1 <= c0) return 0;
    const double w = (double)(c1 - c0);
    const double pairs = w * (double)nrows - (double)(c0 + c1 - 1) * w / 2.0;
    const int prof = lnb_prof_begin(s);
    const int e = lnb_k_tc_syrk_lower(mode == LNB_FACTOR_TF32X3 ? 0 : 1, hi, lo, kstride, nrows, C, ldc, nrows, c0,
                                      c1, k, NULL, st, lnb_wait_ns(), s);
    const double opb = mode == LNB_FACTOR_TF32X3 ? 8.0 : 4.0;
    lnb_prof_end(prof, s, 2.0 * k * pairs, opb * (double)k * ((double)(nrows - c0) + w) + 8.0 * pairs);
    return e;
}

/* block columns j0..j1 of the working matrix from the arrived FP64 data, then
 * the update with panels 0..kdone-1 (K = kdone b) */
static int join_cols(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, const lnb_stream_in *in,
                     const float *HA, const float *LA, int64_t ldk, int j0, int j1, int kdone, cudaStream_t s)
{
    const int64_t c0 = (int64_t)j0 * b, c1 = ((int64_t)j1 + 1) * b < n ? ((int64_t)j1 + 1) * b : n;
    for (int j = j0; j <= j1; ++j) CK(cudaStreamWaitEvent(s, in->arr[j], 0), "arrival wait");
    CK(lnb_k_lower_to_f32_cols(in->A, in->lda, n, c0, c1, in->S, dA, lda, in->rsum, s), "convert");
    if (kdone > 0)
        CK(upd_tc(mode, HA + c0 * ldk, LA ? LA + c0 * ldk : NULL, ldk, dA + c0 + c0 * lda, lda, n - c0, 0, c1 - c0,
                  kdone * b, c->st, s), "catch-up update");
    return 0;
}

/* LNB_UPD_DEPTH: panels a block column beyond the look-ahead collects before it
 * takes them in one update of K = depth b (default 2; 1 updates every step) */
static int upd_depth(void)
{
    const char *e = getenv("LNB_UPD_DEPTH");
    const int v = (e && *e) ? atoi(e) : 2;
    return v < 1 ? 1 : v;
}

/* 0, or the library error for a failed CUDA call */
static int ck_cuda(int err, const char *where) { return err ? lnb_cuda_error(err, where) : 0; }

/* block columns j0..j1 take panels p0..p1 (all of width b) in one update */
static int apply_panels(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, const float *HA, const float *LA,
                        int64_t ldk, int j0, int j1, int p0, int p1, cudaStream_t s)
{
    const int64_t c0 = (int64_t)j0 * b, c1 = ((int64_t)j1 + 1) * b < n ? ((int64_t)j1 + 1) * b : n;
    const int64_t ko = (int64_t)p0 * b;
    CK(upd_tc(mode, HA + c0 * ldk + ko, LA ? LA + c0 * ldk + ko : NULL, ldk, dA + c0 + c0 * lda, lda, n - c0, 0,
              c1 - c0, (p1 - p0 + 1) * b, c->st, s), "panel update");
    return 0;
}

/* inverses of the diagonal blocks of rows [r0, r1) of the factor dA, on the
 * side stream once the critical stream has finished them; r0 and r1 whole
 * 512-blocks (r1 may be n).  Sub-matrices give the same inverses as the whole:
 * the blocks are independent. */
static int blkinv_rows(lnb_ctx *c, const lnb_blkinv *inv, const float *dA, int64_t lda, int64_t n, int64_t r0,
                       int64_t r1)
{
    CK(cudaEventRecord(c->ev[5], c->crit), "event");
    CK(cudaStreamWaitEvent(c->aux, c->ev[5], 0), "event wait");
    const float *T = dA + r0 + r0 * lda;
    float *d64 = inv->dinv64 + (r0 / TRSV_H) * TRSV_H * TRSV_H;
    CK(lnb_k_trtri_blocks_f32(T, lda, r1 - r0, TRSV_H, 'L', 0, d64, c->aux), "trtri");
    if (inv->binv)
        CK(lnb_k_trtri_hb_f32(T, lda, r1 - r0, d64, inv->binv + (r0 / 512) * 512 * 512, c->aux), "block inverses");
    return 0;
}

int lnb_chol_f32_stream_run(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, lnb_refactor_ctx *rf,
                            const lnb_stream_in *in, const lnb_blkinv *inv, lnb_arena *ar, cudaStream_t s)
{
    if (!lnb_chol_f32_stream_ok(n, b, mode)) return lnb_set_error(LNB_EINVAL, "streamed factor: n %d, b %d", n, b);
    const int64_t ldk = ldk_of(n);
    float *dinv = (float *)lnb_arena_take(ar, (size_t)((b + 31) / 32) * 1024 * sizeof(float));
    float *HA = (float *)lnb_arena_take(ar, (size_t)n * ldk * 4);
    float *LA = mode == LNB_FACTOR_TF32X3 ? (float *)lnb_arena_take(ar, (size_t)n * ldk * 4) : NULL;
    if (!dinv || !HA || (mode == LNB_FACTOR_TF32X3 && !LA))
        return lnb_set_error(LNB_ENOMEM, "streamed factor workspace");
    const int mt = (n + b - 1) / b;
    /* u[j]: panels applied to block column j so far (j <= joined) */
    int *u = (int *)calloc((size_t)mt, sizeof(int));
    if (!u) return lnb_set_error(LNB_ENOMEM, "streamed factor: host memory");
    cudaStream_t crit = c->crit;
    cudaEvent_t ev_start = c->ev[0], ev_trsm = c->ev[1], ev_next = c->ev[2], ev_done = c->ev[3];
    cudaEvent_t ev_pace = c->ev[4];
    int e = 0;
    int64_t inv_rows = 0;     /* rows whose diagonal-block inverses are queued on the side stream */
#define RUN(x)                   \
    do {                         \
        if ((e = (x)) != 0) goto out; \
    } while (0)
    RUN(ck_cuda(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset"));
    RUN(ck_cuda(cudaEventRecord(ev_start, s), "event"));
    RUN(ck_cuda(cudaStreamWaitEvent(crit, ev_start, 0), "event wait"));
    {
    const int ahead = stream_ahead() < 0 ? 0 : stream_ahead();
    const int depth = upd_depth();
    /* block columns 0..joined are in the working matrix; without `in` all are */
    int joined = in ? 0 : mt - 1;
    if (in) RUN(join_cols(c, n, b, dA, lda, mode, in, HA, LA, ldk, 0, 0, 0, crit));
    for (int k = 0; k < mt; ++k) {
        const int64_t k0 = (int64_t)k * b;
        const int bs = (int)(n - k0 < b ? n - k0 : b);
        float *Akk = dA + k0 + k0 * lda;
        const int64_t mrem = n - k0 - bs;
        RUN(lnb_potrf_tile_f32(Akk, lda, bs, k0, dinv, c->st, crit));
        if (rf && rf->check) {
            const int info = lnb_status_read(c, crit);
            if (info < 0) { e = info; goto out; }
            if (info > 0) RUN(refactor_tile(c, rf, dA, lda, k0, bs, b, dinv, ar, crit));
        } else if (in) {
            /* keep the host within a step of the device, so the arrival checks
             * below see what has landed, without stalling this step: wait for
             * the previous step's diagonal factor, then queue this step */
            if (k > 0) RUN(ck_cuda(cudaEventSynchronize(ev_pace), "pace"));
            RUN(ck_cuda(cudaEventRecord(ev_pace, crit), "event"));
        }
        if (inv) {
            /* the 512-blocks finished by this step: 8 + 8 small CTAs beside
             * the update, so only the last block's inverse follows the factor */
            const int64_t done = k0 + bs == n ? n : (k0 + bs) / 512 * 512;
            if (done > inv_rows) {
                RUN(blkinv_rows(c, inv, dA, lda, n, inv_rows, done));
                inv_rows = done;
            }
        }
        if (mrem <= 0) break;
        float *hk = HA + (k0 + bs) * ldk + k0, *lk = LA ? LA + (k0 + bs) * ldk + k0 : NULL;
        RUN(ck_cuda(lnb_k_trsm_rlt_prep_f32(Akk, lda, dinv, Akk + bs, lda, mrem, bs, hk, lk, (int)ldk, crit),
                           "trsm+prep f32"));
        RUN(ck_cuda(cudaEventRecord(ev_trsm, crit), "event"));
        /* block columns whose data is here, as far as the host can tell now */
        const int need = k + 2 < mt ? k + 2 : mt - 1;
        int avail = joined;
        if (in) {
            const int cap = need + ahead < mt - 1 ? need + ahead : mt - 1;
            while (avail + 1 <= cap && cudaEventQuery(in->arr[avail + 1]) == cudaSuccess) ++avail;
            cudaGetLastError();   /* cudaErrorNotReady from the queries */
        }
        /* block column k+1 (the next panel), complete through panel k, on the critical stream */
        if (k + 1 > joined) RUN(join_cols(c, n, b, dA, lda, mode, in, HA, LA, ldk, k + 1, k + 1, k + 1, crit));
        else RUN(apply_panels(c, n, b, dA, lda, mode, HA, LA, ldk, k + 1, k + 1, u[k + 1], k, crit));
        u[k + 1] = k + 1;
        RUN(ck_cuda(cudaStreamWaitEvent(s, ev_trsm, 0), "event wait"));
        if (k + 2 < mt) {
            if (k + 2 > joined) RUN(join_cols(c, n, b, dA, lda, mode, in, HA, LA, ldk, k + 2, k + 2, k + 1, s));
            else RUN(apply_panels(c, n, b, dA, lda, mode, HA, LA, ldk, k + 2, k + 2, u[k + 2], k, s));
            u[k + 2] = k + 1;
        }
        RUN(ck_cuda(cudaEventRecord(ev_next, s), "event"));
        /* The other joined columns take their pending panels once `depth` have
         * collected, one launch per run of columns with the same backlog and
         * group.  Blocks of 8 columns belong to groups 0 .. depth-1 in turn;
         * group g takes its first g panels one at a time, so the groups' long
         * updates fall on different steps and the per-step update work stays
         * close to that of one panel for all columns. */
        for (int j = k + 3; j <= joined;) {
            const int g = (j / 8) % depth;
            int j1 = j;
            while (j1 + 1 <= joined && u[j1 + 1] == u[j] && ((j1 + 1) / 8) % depth == g) ++j1;
            if (k + 1 - u[j] >= (k < g ? 1 : depth)) {
                RUN(apply_panels(c, n, b, dA, lda, mode, HA, LA, ldk, j, j1, u[j], k, s));
                for (int q = j; q <= j1; ++q) u[q] = k + 1;
            }
            j = j1 + 1;
        }
        /* newly arrived columns catch up with panels 0..k */
        const int jn = (joined > need ? joined : need) + 1;
        if (avail >= jn) {
            RUN(join_cols(c, n, b, dA, lda, mode, in, HA, LA, ldk, jn, avail, k + 1, s));
            for (int q = jn; q <= avail; ++q) u[q] = k + 1;
        }
        if (need > joined) joined = need;
        if (avail > joined) joined = avail;
        RUN(ck_cuda(cudaStreamWaitEvent(crit, ev_next, 0), "event wait"));
    }
    }
    RUN(ck_cuda(cudaEventRecord(ev_done, crit), "event"));
    RUN(ck_cuda(cudaStreamWaitEvent(s, ev_done, 0), "event wait"));
out:
#undef RUN
    if (inv_rows > 0) {
        /* s (and so whatever reuses this workspace next) follows the side stream */
        int e2 = ck_cuda(cudaEventRecord(c->ev[6], c->aux), "event");
        if (!e2) e2 = ck_cuda(cudaStreamWaitEvent(s, c->ev[6], 0), "event wait");
        if (!e) e = e2;
    }
    free(u);
    return e;
}

/* ---- entry points ---------------------------------------------------------- */
static int check_args(int n, int b, const void *A, int lda)
{
    if (n < 0) return lnb_set_error(LNB_EINVAL, "n = %d < 0", n);
    if (b <= 0 || b > 1024) return lnb_set_error(LNB_EINVAL, "tile size b = %d outside 1..1024", b);
    if (lda < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "lda = %d < n = %d", lda, n);
    if (n > 0 && !A) return lnb_set_error(LNB_EINVAL, "A is NULL");
    return 0;
}

int lnb_schol_dev(int n, int b, float *dA, int lda, int *info_dev, void *stream)
{
    int e = check_args(n, b, dA, lda);
    if (e) return e;
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, lnb_chol_f32_ws_bytes(n, b, g_schol_mode));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    if ((e = lnb_chol_f32_run(c, n, b, dA, lda, g_schol_mode, NULL, &ar, s))) return e;
    if (info_dev) CK(cudaMemcpyAsync(info_dev, &c->st->info, sizeof(int), cudaMemcpyDeviceToDevice, s), "info");
    return 0;
}

static int schol_host(int n, int b, float *A, int lda)
{
    int e = check_args(n, b, A, lda);
    if (e) return e;
    if (n == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ((int64_t)n + 31) & ~(int64_t)31;
    const size_t abytes = (size_t)ldd * n * sizeof(float);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_chol_f32_ws_bytes(n, b, g_schol_mode));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    float *dA = (float *)lnb_arena_take(&ar, abytes);
    cudaStream_t s = c->main;
    for (int64_t c0 = 0; c0 < n; c0 += b) {
        const int64_t w = n - c0 < b ? n - c0 : b;
        CK(cudaMemcpy2DAsync(dA + c0 + c0 * ldd, ldd * sizeof(float), A + c0 + c0 * (int64_t)lda,
                             (size_t)lda * sizeof(float), (size_t)(n - c0) * sizeof(float), w,
                             cudaMemcpyHostToDevice, s), "A in");
    }
    if ((e = lnb_chol_f32_run(c, n, b, dA, ldd, g_schol_mode, NULL, &ar, s))) return e;
    for (int64_t c0 = 0; c0 < n; c0 += b) {
        const int64_t w = n - c0 < b ? n - c0 : b;
        CK(cudaMemcpy2DAsync(A + c0 + c0 * (int64_t)lda, (size_t)lda * sizeof(float), dA + c0 + c0 * ldd,
                             ldd * sizeof(float), (size_t)(n - c0) * sizeof(float), w, cudaMemcpyDeviceToHost, s),
           "L out");
    }
    return lnb_status_read(c, s);
}

int ompss_schol_rl(int n, int b, int t, float *A, int lda) { (void)t; return schol_host(n, b, A, lda); }
int ompss_schol_ll(int n, int b, int t, float *A, int lda) { (void)t; return schol_host(n, b, A, lda); }

static int schol_hyper(int mt, int b, float **Ah)
{
    if (mt < 0 || b <= 0 || b > 1024) return lnb_set_error(LNB_EINVAL, "mt = %d, b = %d", mt, b);
    if (mt == 0) return 0;
    if (!Ah) return lnb_set_error(LNB_EINVAL, "Ah is NULL");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t n = (int64_t)mt * b, ldd = (n + 31) & ~(int64_t)31;
    const size_t abytes = (size_t)ldd * n * sizeof(float);
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_chol_f32_ws_bytes((int)n, b, g_schol_mode));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    float *dA = (float *)lnb_arena_take(&ar, abytes);
    cudaStream_t s = c->main;
    for (int j = 0; j < mt; ++j)
        for (int i = j; i < mt; ++i) {
            if (!Ah[(int64_t)j * mt + i]) return lnb_set_error(LNB_EINVAL, "tile (%d,%d) is NULL", i, j);
            CK(cudaMemcpy2DAsync(dA + (int64_t)i * b + (int64_t)j * b * ldd, ldd * sizeof(float),
                                 Ah[(int64_t)j * mt + i], (size_t)b * sizeof(float), (size_t)b * sizeof(float),
                                 (size_t)b, cudaMemcpyHostToDevice, s), "tile in");
        }
    int e = lnb_chol_f32_run(c, (int)n, b, dA, ldd, g_schol_mode, NULL, &ar, s);
    if (e) return e;
    for (int j = 0; j < mt; ++j)
        for (int i = j; i < mt; ++i)
            CK(cudaMemcpy2DAsync(Ah[(int64_t)j * mt + i], (size_t)b * sizeof(float),
                                 dA + (int64_t)i * b + (int64_t)j * b * ldd, ldd * sizeof(float),
                                 (size_t)b * sizeof(float), (size_t)b, cudaMemcpyDeviceToHost, s), "tile out");
    return lnb_status_read(c, s);
}

int ompss_schol_hrl(int mt, int b, int t, float **Ah) { (void)t; return schol_hyper(mt, b, Ah); }
int ompss_schol_hll(int mt, int b, int t, float **Ah) { (void)t; return schol_hyper(mt, b, Ah); }

/* ---- FP32 solves ---------------------------------------------------------
 * The triangular solves with an FP32 factor compute in FP64 (k_trsv.cu reads
 * the FP32 tiles and accumulates in double); FP32 right-hand sides are
 * widened on the way in and rounded on the way out. */
int lnb_k_f64_to_f32(const double *D, int64_t ldd, int64_t m, int64_t k, float *X, int64_t ldx, cudaStream_t st);

int64_t lnb_trsm_blk_ints(int64_t n);
int64_t lnb_trsm_blk_inv_floats(int64_t n);
int64_t lnb_trsm_blk_vec_doubles(int64_t n, int64_t nrhs);
int lnb_trsm_blk_ok(const float *T, int64_t ldt, int64_t n, int64_t nrhs);
int lnb_k_trsm_blk_f32(char trans, int64_t n, int64_t nrhs, const float *T, int64_t ldt, const float *Binv, double *B,
                       int64_t ldb, double *vec, int *sync, lnb_status_t *st, long long wait_ns, int sms,
                       lnb_stream_t s);

static int spotrs_run(lnb_ctx *c, int64_t n, int64_t nrhs, const float *dL, int64_t lda, float *dB, int64_t ldb,
                      char which, lnb_arena *ar, cudaStream_t s)
{
    const int64_t nb = (n + TRSV_H - 1) / TRSV_H;
    float *dinv = lnb_arena_take(ar, (size_t)nb * TRSV_H * TRSV_H * sizeof(float));
    double *Z = lnb_arena_take(ar, (size_t)n * nrhs * 8);
    int *sync = lnb_arena_take(ar, (size_t)lnb_trsm_sync_ints(n, TRSV_H) * 4);
    if (!sync) return lnb_set_error(LNB_ENOMEM, "spotrs workspace");
    CK(lnb_k_trtri_blocks_f32(dL, lda, n, TRSV_H, 'L', 0, dinv, s), "trtri");
    CK(lnb_k_f32_to_f64(dB, ldb, n, nrhs, Z, n, s), "widen");
    if (lnb_trsm_blk_ok(dL, lda, n, nrhs)) {
        /* few right-hand sides: the solves on the inverses of the large diagonal blocks */
        float *binv = lnb_arena_take(ar, (size_t)lnb_trsm_blk_inv_floats(n) * 4);
        double *vec = lnb_arena_take(ar, (size_t)lnb_trsm_blk_vec_doubles(n, nrhs) * 8);
        int *bsync = lnb_arena_take(ar, (size_t)lnb_trsm_blk_ints(n) * 4);
        if (!bsync) return lnb_set_error(LNB_ENOMEM, "spotrs workspace");
        CK(lnb_k_trtri_hb_f32(dL, lda, n, dinv, binv, s), "block inverses");
        if (which == 'N' || which == 'B')
            CK(lnb_k_trsm_blk_f32('N', n, nrhs, dL, lda, binv, Z, n, vec, bsync, c->st, lnb_wait_ns(), c->sms, s),
               "forward");
        if (which == 'T' || which == 'B')
            CK(lnb_k_trsm_blk_f32('T', n, nrhs, dL, lda, binv, Z, n, vec, bsync, c->st, lnb_wait_ns(), c->sms, s),
               "backward");
        CK(lnb_k_f64_to_f32(Z, n, n, nrhs, dB, ldb, s), "round");
        return 0;
    }
    if (which == 'N' || which == 'B')
        CK(lnb_k_trsm_left_f32('L', 'N', n, nrhs, 1.0, dL, lda, dinv, TRSV_H, Z, n, sync, c->st, lnb_wait_ns(), 0, s),
           "forward");
    if (which == 'T' || which == 'B')
        CK(lnb_k_trsm_left_f32('L', 'T', n, nrhs, 1.0, dL, lda, dinv, TRSV_H, Z, n, sync, c->st, lnb_wait_ns(), 0, s),
           "backward");
    CK(lnb_k_f64_to_f32(Z, n, n, nrhs, dB, ldb, s), "round");
    return 0;
}

static size_t spotrs_ws_bytes(int64_t n, int64_t nrhs)
{
    const int64_t nb = (n + TRSV_H - 1) / TRSV_H;
    return lnb_align256((size_t)nb * TRSV_H * TRSV_H * 8) + lnb_align256((size_t)n * nrhs * 8) +
           lnb_align256((size_t)lnb_trsm_sync_ints(n, TRSV_H) * 4) + lnb_align256((size_t)lnb_trsm_blk_inv_floats(n) * 4) +
           lnb_align256((size_t)lnb_trsm_blk_vec_doubles(n, nrhs) * 8) + lnb_align256((size_t)lnb_trsm_blk_ints(n) * 4) +
           1024;
}

int lnb_spotrs_dev(int n, int nrhs, const float *dL, int lda, float *dB, int ldb, char which, void *stream)
{
    if (n < 0 || nrhs < 0 || lda < (n > 1 ? n : 1) || ldb < (n > 1 ? n : 1))
        return lnb_set_error(LNB_EINVAL, "spotrs sizes");
    if (which != 'N' && which != 'T' && which != 'B') return lnb_set_error(LNB_EINVAL, "spotrs which");
    if (n == 0 || nrhs == 0) return 0;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    void *ws = lnb_ws(c, spotrs_ws_bytes(n, nrhs));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemsetAsync(c->st, 0, sizeof(lnb_status_t), s), "status reset");
    return spotrs_run(c, n, nrhs, dL, lda, dB, ldb, which, &ar, s);
}

/* sspdsolv_main (spdsolv_main.c:10-20 built with -DSINGLE_PRECISION) */
int sspdsolv_main(int m, int nrhs, int b, float *A, float *B)
{
    if (m < 0 || nrhs < 0 || b <= 0 || b > 1024) return lnb_set_error(LNB_EINVAL, "spdsolv arguments");
    if (m == 0) return 0;
    if (!A || (nrhs > 0 && !B)) return lnb_set_error(LNB_EINVAL, "NULL matrix");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int64_t ldd = ((int64_t)m + 31) & ~(int64_t)31;
    const size_t abytes = (size_t)ldd * m * 4, bbytes = (size_t)ldd * (nrhs ? nrhs : 1) * 4;
    void *ws = lnb_ws(c, lnb_align256(abytes) + lnb_align256(bbytes) + lnb_chol_f32_ws_bytes(m, b, g_schol_mode) +
                             spotrs_ws_bytes(m, nrhs ? nrhs : 1));
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    float *dA = lnb_arena_take(&ar, abytes), *dB = lnb_arena_take(&ar, bbytes);
    cudaStream_t s = c->main;
    for (int64_t c0 = 0; c0 < m; c0 += b) {
        const int64_t w = m - c0 < b ? m - c0 : b;
        CK(cudaMemcpy2DAsync(dA + c0 + c0 * ldd, ldd * 4, A + c0 + c0 * (int64_t)m, (size_t)m * 4,
                             (size_t)(m - c0) * 4, w, cudaMemcpyHostToDevice, s), "A in");
    }
    if (nrhs > 0)
        CK(cudaMemcpy2DAsync(dB, ldd * 4, B, (size_t)m * 4, (size_t)m * 4, nrhs, cudaMemcpyHostToDevice, s), "B in");
    lnb_arena ar2 = ar;
    int e = lnb_chol_f32_run(c, m, b, dA, ldd, g_schol_mode, NULL, &ar2, s);
    if (e) return e;
    if (nrhs > 0) {
        if ((e = spotrs_run(c, m, nrhs, dA, ldd, dB, ldd, 'B', &ar, s))) return e;
        CK(cudaMemcpy2DAsync(B, (size_t)m * 4, dB, ldd * 4, (size_t)m * 4, nrhs, cudaMemcpyDeviceToHost, s), "X out");
    }
    for (int64_t c0 = 0; c0 < m; c0 += b) {
        const int64_t w = m - c0 < b ? m - c0 : b;
        CK(cudaMemcpy2DAsync(A + c0 + c0 * (int64_t)m, (size_t)m * 4, dA + c0 + c0 * ldd, ldd * 4,
                             (size_t)(m - c0) * 4, w, cudaMemcpyDeviceToHost, s), "L out");
    }
    return lnb_status_read(c, s);
}
