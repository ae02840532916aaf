/*
 * lnb_host.h -- internal declarations shared by the host-side C files.
 */
#ifndef LNB_HOST_H
#define LNB_HOST_H

#include <cuda_runtime_api.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/linompss_b200.h"
#include "lnb_kern.h"

#ifdef __cplusplus
extern "C" {
#endif

/* per-device context: streams, events, cached workspace, status words */
typedef struct {
    int           ready;
    int           device;
    int           sms;
    cudaStream_t  main;        /* stream of the host-pointer entry points */
    cudaStream_t  crit;        /* high-priority stream: panel factorization */
    cudaStream_t  copy;        /* device->host panel copies */
    cudaStream_t  aux;         /* low-priority stream: work beside the critical path */
    cudaEvent_t   ev[8];
    void         *ws;          /* grow-only device workspace */
    size_t        ws_size;
    lnb_status_t *st;          /* device status word */
    lnb_status_t *st_host;     /* pinned host mirror */
    cudaEvent_t   t0, t1;      /* timing */
} lnb_ctx;

/* Returns the current device's context (creating it), or NULL after setting
 * the error (LNB_ENODEV / LNB_ECUDA). */
lnb_ctx *lnb_ctx_get(void);
/* Ensure the cached workspace holds at least `bytes`; NULL on failure. */
void *lnb_ws(lnb_ctx *c, size_t bytes);

/* workspace carving: bump allocator over one buffer, 256-byte aligned */
typedef struct { char *base; size_t off, cap; } lnb_arena;
static inline size_t lnb_align256(size_t x) { return (x + 255) & ~(size_t)255; }
static inline void *lnb_arena_take(lnb_arena *a, size_t bytes)
{
    size_t o = lnb_align256(a->off);
    if (o + bytes > a->cap) return NULL;
    a->off = o + bytes;
    return a->base + o;
}

int  lnb_set_error(int code, const char *fmt, ...);
int  lnb_cuda_error(int cuda_err, const char *where);
long long lnb_wait_ns(void);

/* Read back the status word after the stream work completed; returns info
 * (>= 0) or LNB_ETIMEOUT.  Synchronizes `s`. */
int lnb_status_read(lnb_ctx *c, cudaStream_t s);

/* ---- FP64 factorization schedule on device memory (lnb_chol.c) ---------- */
/* one diagonal tile (bs <= 1024): leaf kernel or nested 128-wide pass; fills
 * dinv with the inverses of its 32x32 diagonal blocks */
int lnb_potrf_tile_f64(double *Akk, int64_t lda, int bs, int64_t row0, double *dinv,
                       lnb_status_t *st, cudaStream_t s);
size_t lnb_chol_f64_ws_bytes(int n, int b);
/* Factor dA in place on stream s.  `copy_back` (may be NULL): host matrix to
 * receive each finished panel as soon as it is final (lower part). */
int lnb_chol_f64_run(lnb_ctx *c, int n, int b, double *dA, int64_t lda, lnb_arena *ar,
                     cudaStream_t s, double *copy_back, int64_t ldh);

/* the schedule the FP64 factorization of order n runs: 1 device DAG, 0 streams */
int lnb_chol_f64_uses_dag(int n);
/* Factor with the chosen schedule.  w_out (may be NULL) receives the device
 * DAG's 64 x 64 diagonal-block inverses of L (the triangular solves' layout),
 * or NULL when the stream schedule ran. */
int lnb_chol_f64_run_w(lnb_ctx *c, int n, int b, double *dA, int64_t lda, lnb_arena *ar, cudaStream_t s,
                       double *copy_back, int64_t ldh, double **w_out);

/* ---- FP32-storage factorization (lnb_chol32.c) ---------------------------- */
int lnb_potrf_tile_f32(float *Akk, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                       cudaStream_t s);
size_t lnb_chol_f32_ws_bytes(int n, int b, int mode);
/* FP64 diagonal-tile refactor context: when passed to lnb_chol_f32_run, a
 * diagonal tile whose low-precision pivot is not positive is rebuilt from
 * the original FP64 matrix (lower part, equilibration S) and refactored in
 * FP64; the arena must then also hold lnb_refactor_ws_bytes(b). */
typedef struct {
    const double *A;
    int64_t lda;
    const double *S;
    int refactored, shifted;
    /* 1: read the status after every diagonal tile and refactor a failed one
     * at once (a host round trip per step); 0: no per-step reads -- the caller
     * checks the final status and reruns with 1 if a pivot failed */
    int check;
} lnb_refactor_ctx;
size_t lnb_refactor_ws_bytes(int b);
int lnb_chol_f32_run(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, lnb_refactor_ctx *rf,
                     lnb_arena *ar, cudaStream_t s);
int lnb_get_factor_mode(void);
/* A matrix arriving block column by block column on another stream: block
 * column j (columns [j b, (j+1) b), rows >= j b) of the FP64 copy A is
 * complete once arr[j] has fired; S is the equilibration scale on the device;
 * rsum (NULL, or n zeroed doubles) gains the row sums of |A| as the block
 * columns are converted. */
typedef struct {
    const double *A;
    int64_t lda;
    const double *S;
    cudaEvent_t *arr;
    double *rsum;
} lnb_stream_in;
int lnb_chol_f32_stream_ok(int n, int b, int mode);
size_t lnb_chol_f32_stream_ws_bytes(int n, int b, int mode);
/* Inverses of the factor's diagonal blocks for the triangular solves that
 * follow: the 64 x 64 ones into dinv64 (lnb_k_trtri_blocks_f32) and, when binv
 * is not NULL, the 512 x 512 ones (lnb_k_trtri_hb_f32). */
typedef struct {
    float *dinv64;
    float *binv;
} lnb_blkinv;
/* The FP32 factorization of lower(S A S) into dA, keeping every panel's
 * operand copies: while A arrives (in != NULL, dA filled block column by block
 * column), or with dA already complete (in == NULL).  With inv != NULL the
 * diagonal-block inverses are formed on the side stream as the diagonal tiles
 * are finished, and are complete on s when the call's work is. */
int lnb_chol_f32_stream_run(lnb_ctx *c, int n, int b, float *dA, int64_t lda, int mode, lnb_refactor_ctx *rf,
                            const lnb_stream_in *in, const lnb_blkinv *inv, lnb_arena *ar, cudaStream_t s);

/* ---- FP64 triangular solves on device memory (lnb_solve.c) --------------- */
size_t lnb_trsm_f64_ws_bytes(int64_t n, int64_t nrhs);
int lnb_trsm_f64_run(lnb_ctx *c, char uplo, char trans, char diag, int64_t n, int64_t nrhs,
                     double alpha, const double *dT, int64_t ldt, double *dB, int64_t ldb,
                     lnb_arena *ar, cudaStream_t s, const double *dinv_given);

/* diagnostics: bracket one launch with events when profiling is on */
int  lnb_prof_begin(cudaStream_t s);
void lnb_prof_end(int slot, cudaStream_t s, double flops, double bytes);

/* is this host pointer page-locked (so async copies really are async)? */
int lnb_host_is_pinned(const void *p);

#ifdef __cplusplus
}
#endif
#endif
