/*
 * lnb_batched.c -- batched uneven SPD solves (host C).
 *
 * One call = two launches on the caller's stream: a device-side counting sort
 * of the systems by size (largest first) and the persistent solver
 * (k_batched.cu).  Nothing synchronizes the host, so the call can be
 * captured in a CUDA graph once the workspace exists (any earlier call, or
 * lnb_batched_autotune, creates it).
 *
 * Autotuning: lnb_batched_autotune times the candidate launch shapes on the
 * caller's own batch and keeps the fastest for the rest of the process:
 *   - CTA size (256 or 512 threads),
 *   - resident systems per SM (1 or 2: two 256-thread FP32 CTAs fit one SM's
 *     shared memory and registers, so one system's latency chain hides the
 *     other's),
 *   - processing order (largest first, or largest/smallest interleaved).
 * FP64 mode's panel fills the shared memory: one 256-thread CTA per SM, both
 * orders.
 */
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

size_t lnb_batched_scratch_bytes(int grid, int fp64);
int lnb_k_batched_posv(int count, const int *n, const int *nrhs, const int64_t *a_off, const int64_t *b_off,
                       const double *A, const double *B, double *X, void *scratch, int grid, const int *order,
                       int *ticket, int *info, int *iters, int max_iter, int fp64, int variant, cudaStream_t s);
int lnb_k_batch_order(int count, const int *n, int *order, int interleave, cudaStream_t s);

#define CK(call, where)                                            \
    do {                                                           \
        int _e = (int)(call);                                      \
        if (_e != 0) return lnb_cuda_error(_e, where);             \
    } while (0)

typedef struct { int nt, per_sm, interleave; } bcfg;
static bcfg g_cfg[2] = {{256, 1, 0}, {256, 1, 0}};   /* tuned shape: [fp32 mode, fp64 mode] */

static int batched_run(int count, const int *n, const int *nrhs, const int64_t *a_off, const int64_t *b_off,
                       const double *dA, const double *dB, double *dX, int mode, int max_iter, int *info,
                       int *iters, cudaStream_t s, bcfg cf)
{
    if (count < 0) return lnb_set_error(LNB_EINVAL, "count = %d < 0", count);
    if (count == 0) return 0;
    if (!n || !nrhs || !a_off || !b_off || !dA || !dB || !dX) return lnb_set_error(LNB_EINVAL, "NULL argument");
    if (mode != LNB_FACTOR_FP32 && mode != LNB_FACTOR_FP64)
        return lnb_set_error(LNB_EINVAL, "batched: mode must be LNB_FACTOR_FP32 or LNB_FACTOR_FP64");
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    const int fp64 = mode == LNB_FACTOR_FP64;
    const int grid = c->sms * cf.per_sm;
    const size_t sb = lnb_batched_scratch_bytes(grid, fp64);
    void *ws = lnb_ws(c, lnb_align256(sb) + lnb_align256((size_t)count * 4) + 512);
    if (!ws) return LNB_ENOMEM;
    lnb_arena ar = {(char *)ws, 0, c->ws_size};
    void *scratch = lnb_arena_take(&ar, sb);
    int *order = lnb_arena_take(&ar, (size_t)count * 4);
    int *ticket = lnb_arena_take(&ar, 64);
    if (!ticket) return lnb_set_error(LNB_ENOMEM, "batched workspace");
    CK(lnb_k_batch_order(count, n, order, cf.interleave, s), "order");
    CK(lnb_k_batched_posv(count, n, nrhs, a_off, b_off, dA, dB, dX, scratch, grid, order, ticket, info, iters,
                          max_iter > 0 ? max_iter : 10, fp64, cf.nt, s), "batched");
    return 0;
}

int lnb_batched_posv_dev(int count, const int *n_dev, const int *nrhs_dev, const int64_t *a_off_dev,
                         const int64_t *b_off_dev, const double *dA, const double *dB, double *dX, int mode,
                         int max_iter, int *info_dev, int *iters_dev, void *stream)
{
    return batched_run(count, n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode, max_iter, info_dev,
                       iters_dev, (cudaStream_t)stream, g_cfg[mode == LNB_FACTOR_FP64]);
}

int lnb_batched_config(int mode, int *cta_threads, int *ctas_per_sm, int *interleave)
{
    const bcfg cf = g_cfg[mode == LNB_FACTOR_FP64];
    if (cta_threads) *cta_threads = cf.nt;
    if (ctas_per_sm) *ctas_per_sm = cf.per_sm;
    if (interleave) *interleave = cf.interleave;
    return 0;
}

int lnb_batched_autotune(int count, const int *n_dev, const int *nrhs_dev, const int64_t *a_off_dev,
                         const int64_t *b_off_dev, const double *dA, const double *dB, double *dX, int mode,
                         int max_iter, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    lnb_ctx *c = lnb_ctx_get();
    if (!c) return LNB_ENODEV;
    static const bcfg cand32[] = {{256, 1, 0}, {256, 2, 0}, {256, 2, 1}, {512, 1, 0}, {512, 1, 1}};
    static const bcfg cand64[] = {{256, 1, 0}, {256, 1, 1}};
    const bcfg *cand = mode == LNB_FACTOR_FP64 ? cand64 : cand32;
    const int ncand = mode == LNB_FACTOR_FP64 ? 2 : 5;
    float best = 1e30f;
    bcfg pick = cand[0];
    for (int k = 0; k < ncand; ++k) {
        for (int rep = 0; rep < 2; ++rep) {   /* first run warms up */
            CK(cudaEventRecord(c->t0, s), "event");
            int e = batched_run(count, n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode, max_iter, NULL,
                                NULL, s, cand[k]);
            if (e) return e;
            CK(cudaEventRecord(c->t1, s), "event");
            CK(cudaEventSynchronize(c->t1), "sync");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->t0, c->t1);
            if (rep == 1 && ms < best) {
                best = ms;
                pick = cand[k];
            }
        }
    }
    g_cfg[mode == LNB_FACTOR_FP64] = pick;
    return pick.nt;
}

/* ---- multi-GPU split of a batch -------------------------------------------- */
typedef struct { double cost; int idx; } part_item;

static int part_cmp(const void *a, const void *b)
{
    const part_item *x = (const part_item *)a, *y = (const part_item *)b;
    if (x->cost != y->cost) return x->cost > y->cost ? -1 : 1;
    return x->idx - y->idx;
}

int lnb_batched_partition(int count, const int *n, const int *nrhs, int parts, int *owner, double *load)
{
    if (count < 0 || parts <= 0 || (count > 0 && (!n || !nrhs || !owner)))
        return lnb_set_error(LNB_EINVAL, "batched partition: count %d, parts %d", count, parts);
    double *acc = (double *)calloc((size_t)parts, sizeof(double));
    part_item *it = (part_item *)malloc((size_t)(count > 0 ? count : 1) * sizeof(part_item));
    if (!acc || !it) {
        free(acc);
        free(it);
        return lnb_set_error(LNB_ENOMEM, "batched partition: host memory");
    }
    for (int s = 0; s < count; ++s) {
        const double ns = (double)n[s], rs = (double)nrhs[s];
        it[s].cost = ns * ns * ns / 3.0 + 2.0 * ns * ns * rs;
        it[s].idx = s;
    }
    qsort(it, (size_t)count, sizeof(part_item), part_cmp);
    for (int k = 0; k < count; ++k) {
        int best = 0;
        for (int p = 1; p < parts; ++p)
            if (acc[p] < acc[best]) best = p;
        owner[it[k].idx] = best;
        acc[best] += it[k].cost;
    }
    if (load) memcpy(load, acc, (size_t)parts * sizeof(double));
    free(acc);
    free(it);
    return 0;
}
