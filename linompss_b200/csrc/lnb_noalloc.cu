// lnb_noalloc.cu -- FP64 tile Cholesky that allocates no device memory.
//
// Who needs this: a caller whose device memory is owned by another manager
// (a caching allocator or a fixed arena that holds the whole HBM), or a
// caller on a latency-critical path where cudaMalloc's implicit device
// synchronization is not acceptable.  Such callers cannot let the library
// grow its cached workspace or create its per-device context (which
// allocates a status word and pinned host memory).
//
// lnb_dchol_noalloc_dev therefore keeps its only scratch -- the inverses of
// the 32x32 diagonal blocks of the current tile and the status word -- in
// one file-scope __device__ array of fixed size, runs every kernel on the
// caller's stream (no look-ahead stream, no events), and calls no allocating
// routine.  Every GPU that loads the library holds that array until the
// process exits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "lnb_host.h"

// inverses for tiles up to LNB_NOALLOC_MAX_B (32 blocks of 32 x 32 doubles),
// then the status word, rounded up to whole doubles
#define LNB_NOALLOC_MAX_B 1024
#define LNB_NOALLOC_DINV ((LNB_NOALLOC_MAX_B / 32) * 1024)
#define LNB_NOALLOC_STATUS ((sizeof(lnb_status_t) + sizeof(double) - 1) / sizeof(double))
static __device__ __align__(256) double g_noalloc_scratch[LNB_NOALLOC_DINV + LNB_NOALLOC_STATUS];
static_assert(sizeof(g_noalloc_scratch) >= LNB_NOALLOC_DINV * sizeof(double) + sizeof(lnb_status_t),
              "the status word must fit behind the block inverses");

// device address of g_noalloc_scratch, looked up once per device with that
// device current (a host-side reference to the symbol is not a device address).
// The cached address lives as long as the device's primary context: a
// cudaDeviceReset in the caller's process makes it stale.
static double *g_scratch_dev[64];

static int scratch_for_current_device(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return lnb_set_error(LNB_ENODEV, "no CUDA device: %s", cudaGetErrorString(e));
    if (!g_scratch_dev[dev]) {
        void *p = NULL;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return lnb_cuda_error(e, "cudaGetSymbolAddress(scratch)");
        g_scratch_dev[dev] = (double *)p;
    }
    *out = g_scratch_dev[dev];
    return 0;
}

extern "C" int lnb_dchol_noalloc_dev(int n, int b, double *dA, int lda, int *info_dev, void *stream)
{
    if (n < 0) return lnb_set_error(LNB_EINVAL, "n = %d < 0", n);
    if (b <= 0) return lnb_set_error(LNB_EINVAL, "tile size b = %d <= 0", b);
    if (b > LNB_NOALLOC_MAX_B)
        return lnb_set_error(LNB_ETOOBIG, "lnb_dchol_noalloc_dev: tile size b = %d exceeds the fixed scratch "
                                          "limit of %d", b, LNB_NOALLOC_MAX_B);
    if (lda < (n > 1 ? n : 1)) return lnb_set_error(LNB_EINVAL, "lda = %d < n = %d", lda, n);
    if (n > 0 && !dA) return lnb_set_error(LNB_EINVAL, "A is NULL");
    if (n == 0) return 0;
    double *scratch = NULL;
    int e = scratch_for_current_device(&scratch);
    if (e) return e;
    double *dinv = scratch;
    lnb_status_t *st = (lnb_status_t *)(scratch + LNB_NOALLOC_DINV);
    cudaStream_t s = (cudaStream_t)stream;
    // the array keeps the previous call's contents: the status word must start at zero
    cudaError_t ce = cudaMemsetAsync(st, 0, sizeof(lnb_status_t), s);
    if (ce != cudaSuccess) return lnb_cuda_error(ce, "status reset");
    const int mt = (n + b - 1) / b;
    for (int k = 0; k < mt; ++k) {
        const int64_t k0 = (int64_t)k * b;
        const int bs = (int)(n - k0 < b ? n - k0 : b);
        double *Akk = dA + k0 + k0 * (int64_t)lda;
        const int64_t mrem = n - k0 - bs;
        if ((e = lnb_potrf_tile_f64(Akk, lda, bs, k0, dinv, st, s))) return e;
        if (mrem <= 0) break;
        if ((e = lnb_k_trsm_rlt_f64(Akk, lda, dinv, Akk + bs, lda, mrem, bs, s)))
            return lnb_cuda_error(e, "trsm");
        if ((e = lnb_k_syrk_lower_f64(Akk + bs, lda, Akk + bs + (int64_t)bs * lda, lda, mrem, 0, mrem, bs, s)))
            return lnb_cuda_error(e, "update");
    }
    if (info_dev) {
        ce = cudaMemcpyAsync(info_dev, &st->info, sizeof(int), cudaMemcpyDeviceToDevice, s);
        if (ce != cudaSuccess) return lnb_cuda_error(ce, "info");
    }
    return 0;
}
