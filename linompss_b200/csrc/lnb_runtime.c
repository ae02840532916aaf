/*
 * lnb_runtime.c -- device contexts, workspace cache, errors, status words.
 *
 * The reference has no runtime of its own beyond the OmpSs task system
 * (Nanos++), which this library replaces with explicit CUDA streams (panel
 * work on a high-priority stream, trailing updates on the caller's stream)
 * and device-side DAG walks.  Everything here is host C.
 */
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lnb_host.h"

#define LNB_MAX_DEV 16

static lnb_ctx g_ctx[LNB_MAX_DEV];
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
static __thread char t_err[512] = "no error";
static long long g_wait_ns = 2000000000LL;  /* 2 s of device time */

const char *lnb_version(void) { return "linompss-b200 0.1 (sm_100a)"; }
const char *lnb_last_error(void) { return t_err; }

int lnb_set_error(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof t_err, fmt, ap);
    va_end(ap);
    return code;
}

int lnb_cuda_error(int e, const char *where)
{
    if (e == cudaErrorMemoryAllocation)
        return lnb_set_error(LNB_ENOMEM, "%s: %s", where, cudaGetErrorString((cudaError_t)e));
    return lnb_set_error(LNB_ECUDA, "%s: %s", where, cudaGetErrorString((cudaError_t)e));
}

void lnb_set_wait_limit_us(long long us) { g_wait_ns = us > 0 ? us * 1000LL : 2000000000LL; }
long long lnb_wait_ns(void) { return g_wait_ns; }

lnb_ctx *lnb_ctx_get(void)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= LNB_MAX_DEV) {
        lnb_set_error(LNB_ENODEV, "no CUDA device: %s", cudaGetErrorString(e));
        return NULL;
    }
    lnb_ctx *c = &g_ctx[dev];
    if (c->ready) return c;
    pthread_mutex_lock(&g_lock);
    if (!c->ready) {
        struct cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major != 10) {
            pthread_mutex_unlock(&g_lock);
            lnb_set_error(LNB_ENODEV, "device %d is not sm_100 (compute %d.%d); this library "
                          "runs on B200 only", dev, prop.major, prop.minor);
            return NULL;
        }
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        int ok = cudaStreamCreateWithPriority(&c->crit, cudaStreamNonBlocking, hi) == cudaSuccess &&
                 cudaStreamCreateWithFlags(&c->main, cudaStreamNonBlocking) == cudaSuccess &&
                 cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) == cudaSuccess &&
                 cudaStreamCreateWithPriority(&c->aux, cudaStreamNonBlocking, lo) == cudaSuccess;
        for (int i = 0; ok && i < 8; ++i)
            ok = cudaEventCreateWithFlags(&c->ev[i], cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaEventCreate(&c->t0) == cudaSuccess && cudaEventCreate(&c->t1) == cudaSuccess;
        ok = ok && cudaMalloc((void **)&c->st, sizeof(lnb_status_t)) == cudaSuccess;
        ok = ok && cudaMallocHost((void **)&c->st_host, sizeof(lnb_status_t)) == cudaSuccess;
        if (!ok) {
            pthread_mutex_unlock(&g_lock);
            lnb_set_error(LNB_ECUDA, "context setup failed on device %d", dev);
            return NULL;
        }
        c->device = dev;
        c->sms = prop.multiProcessorCount;
        c->ready = 1;
    }
    pthread_mutex_unlock(&g_lock);
    return c;
}

void *lnb_ws(lnb_ctx *c, size_t bytes)
{
    if (bytes <= c->ws_size && c->ws) return c->ws;
    if (c->ws) {
        cudaDeviceSynchronize();
        cudaFree(c->ws);
        c->ws = NULL;
        c->ws_size = 0;
    }
    size_t want = bytes + bytes / 8 + (1 << 20);
    if (cudaMalloc(&c->ws, want) != cudaSuccess) {
        cudaGetLastError();
        c->ws = NULL;
        lnb_set_error(LNB_ENOMEM, "workspace of %zu bytes", want);
        return NULL;
    }
    c->ws_size = want;
    return c->ws;
}

void lnb_release_workspace(void)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= LNB_MAX_DEV) return;
    lnb_ctx *c = &g_ctx[dev];
    if (c->ready && c->ws) {
        cudaDeviceSynchronize();
        cudaFree(c->ws);
        c->ws = NULL;
        c->ws_size = 0;
    }
}

int lnb_status_read(lnb_ctx *c, cudaStream_t s)
{
    cudaError_t e = cudaMemcpyAsync(c->st_host, c->st, sizeof(lnb_status_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return lnb_cuda_error(e, "status read");
    if (c->st_host->timeout)
        return lnb_set_error(LNB_ETIMEOUT, "device-side dependency wait ran out (site %d, item %d)",
                             c->st_host->timeout, c->st_host->timeout_item);
    return c->st_host->info;
}

/* ---- diagnostics: launch counts and timed update launches ----------------- */
#define PROF_MAX 8192
static struct {
    int on;
    long long launches;
    int npairs;
    cudaEvent_t ev[PROF_MAX][2];
    double flops[PROF_MAX], bytes[PROF_MAX];
    long long done_launches;
    double done_ms, done_flops, done_bytes;
} g_prof;

void lnb_prof_count(int k) { g_prof.launches += k; }
void lnb_prof_enable(int on) { g_prof.on = on; }

static void prof_drain(void)
{
    for (int i = 0; i < g_prof.npairs; ++i) {
        float ms = 0.f;
        cudaEventSynchronize(g_prof.ev[i][1]);
        cudaEventElapsedTime(&ms, g_prof.ev[i][0], g_prof.ev[i][1]);
        g_prof.done_ms += ms;
        g_prof.done_flops += g_prof.flops[i];
        g_prof.done_bytes += g_prof.bytes[i];
        g_prof.done_launches += 1;
    }
    g_prof.npairs = 0;
}

void lnb_prof_reset(void)
{
    prof_drain();
    g_prof.launches = 0;
    g_prof.done_launches = 0;
    g_prof.done_ms = g_prof.done_flops = g_prof.done_bytes = 0.0;
}

int lnb_prof_read(lnb_prof_t *out)
{
    prof_drain();
    if (!out) return LNB_EINVAL;
    out->launches = g_prof.launches;
    out->update_launches = g_prof.done_launches;
    out->update_ms = g_prof.done_ms;
    out->update_flops = g_prof.done_flops;
    out->update_bytes = g_prof.done_bytes;
    return 0;
}

int lnb_prof_begin(cudaStream_t s)
{
    if (!g_prof.on) return -1;
    if (g_prof.npairs >= PROF_MAX) prof_drain();
    int i = g_prof.npairs;
    if (!g_prof.ev[i][0]) {
        cudaEventCreate(&g_prof.ev[i][0]);
        cudaEventCreate(&g_prof.ev[i][1]);
    }
    cudaEventRecord(g_prof.ev[i][0], s);
    return i;
}

void lnb_prof_end(int i, cudaStream_t s, double flops, double bytes)
{
    if (i < 0) return;
    cudaEventRecord(g_prof.ev[i][1], s);
    g_prof.flops[i] = flops;
    g_prof.bytes[i] = bytes;
    g_prof.npairs = i + 1;
}

int lnb_host_is_pinned(const void *p)
{
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost;
}
