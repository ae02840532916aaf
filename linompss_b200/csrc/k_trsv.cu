// k_trsv.cu -- blocked triangular solves with many or few right-hand sides.
//
// Semantics of bblas_dltrsm (bblas_trsm.h:116-202) and of the two solves of
// dspdsolv_main (spdsolv_main.c:15,17): op(T) X = alpha B with T triangular.
//
// Design: the reference walks block rows with one TRSM task per diagonal
// block and one GEMM task per off-diagonal block.  Here the same task DAG
// runs inside ONE persistent launch:
//   * the h x h diagonal blocks are inverted up front (k_trtri_blocks), so a
//     diagonal "task" is a small GEMM X_j = inv(T_jj) B_j instead of a
//     sequential substitution;
//   * CTAs take work items from an atomic ticket in DAG order (column j's
//     diagonal item, then its off-diagonal updates B_i -= T_ij X_j), so every
//     item only ever waits on items with smaller tickets, which are already
//     held by running CTAs -- the walk cannot deadlock whatever the CTA
//     scheduling order;
//   * an update item stages its T tile in shared memory BEFORE waiting on
//     X_j, so the HBM stream of T overlaps the dependency chain;
//   * every wait is bounded (globaltimer) and reports a timeout instead of
//     hanging.
// Both the tile products use DMMA (m16n8k4 f64).
#include "common.cuh"

namespace lnb {

constexpr int TH = 64;          // block size
constexpr int TLD = TH + 4;     // k-major smem stride (= 4 mod 16 doubles)
constexpr int NRC = 64;         // rhs columns per pass

// ------------------------------------------------------------------------
// inverses of the diagonal blocks
// ------------------------------------------------------------------------
template <typename TT>
__global__ void __launch_bounds__(TH) k_trtri_blocks(const TT *T, int64_t ldt, int64_t n, char uplo, int unit,
                                                     double *dinv)
{
    extern __shared__ double smx[];
    double (*X)[TH + 1] = reinterpret_cast<double (*)[TH + 1]>(smx);              // X[r][c], column c owned by thread c
    double (*Tb)[TH + 1] = reinterpret_cast<double (*)[TH + 1]>(smx + TH * (TH + 1));
    const int q = blockIdx.x, c = threadIdx.x;
    const int64_t o = (int64_t)q * TH;
    const int qn = (int)((n - o) < TH ? (n - o) : TH);
    for (int r = 0; r < TH; ++r) {
        double v = 0.0;
        if (r < qn && c < qn) v = (double)T[(o + r) + (o + c) * ldt];
        Tb[r][c] = v;
    }
    __syncthreads();
    for (int r = 0; r < TH; ++r) X[r][c] = 0.0;
    if (c >= qn) {
        X[c][c] = 1.0;
    } else if (uplo == 'L') {
        // column c of inv(L): x[c] = 1/L[c][c]; x[r] = -(sum_{p=c}^{r-1} L[r][p] x[p]) / L[r][r]
        X[c][c] = unit ? 1.0 : 1.0 / Tb[c][c];
        for (int r = c + 1; r < qn; ++r) {
            double s = 0.0;
            for (int p = c; p < r; ++p) s += Tb[r][p] * X[p][c];
            X[r][c] = unit ? -s : -s / Tb[r][r];
        }
    } else {
        // column c of inv(U): x[c] = 1/U[c][c]; x[r] = -(sum_{p=r+1}^{c} U[r][p] x[p]) / U[r][r]
        X[c][c] = unit ? 1.0 : 1.0 / Tb[c][c];
        for (int r = c - 1; r >= 0; --r) {
            double s = 0.0;
            for (int p = r + 1; p <= c; ++p) s += Tb[r][p] * X[p][c];
            X[r][c] = unit ? -s : -s / Tb[r][r];
        }
    }
    __syncthreads();
    double *D = dinv + (int64_t)q * TH * TH;
    for (int r = 0; r < TH; ++r) D[r + TH * c] = X[r][c];
}

// ------------------------------------------------------------------------
// the DAG walk
// ------------------------------------------------------------------------
template <typename TT>
struct TrsmArgs {
    const TT *T; int64_t ldt; const double *dinv;
    double *B; int64_t ldb; int64_t n, nrhs;
    int nb; int fwd; int tT;   // tT: op(T) = T^T
    int *ticket, *cnt, *ready;
    lnb_status_t *st; long long wait_ns;
};

// acc(16 rows of warp w, NRC cols) = A(TH x TH, k-major smem) * Bm(TH x NRC, k-major smem)
LNB_DEV void tile_mma(const double *As, const double *Bs, double (&acc)[NRC / 8][4], int w, int g,
                      int t, int ntiles)
{
#pragma unroll
    for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[ni][q] = 0.0;
#pragma unroll 4
    for (int kq = 0; kq < TH / 4; ++kq) {
        const double a0 = As[(kq * 4 + t) * TLD + w * 16 + g];
        const double a1 = As[(kq * 4 + t) * TLD + w * 16 + g + 8];
#pragma unroll
        for (int ni = 0; ni < NRC / 8; ++ni)
            if (ni < ntiles) dmma16x8x4(acc[ni], a0, a1, Bs[(kq * 4 + t) * TLD + ni * 8 + g]);
    }
}

template <typename TT>
__global__ void __launch_bounds__(128) k_trsm_dag(TrsmArgs<TT> a)
{
    extern __shared__ double smd[];
    double *As = smd;              // [TH][TLD]
    double *Bs = smd + TH * TLD;   // [TH][TLD]
    __shared__ int s_item, s_ok;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
    const int nb = a.nb;
    const int64_t total = (int64_t)nb * (nb + 1) / 2;

    while (true) {
        if (tid == 0) s_item = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int64_t item = s_item;
        __syncthreads();
        if (item >= total) break;

        // decode: virtual column jj starts at S(jj) = jj*nb - jj*(jj-1)/2
        const double B2 = 2.0 * nb + 1.0;
        int jj = (int)((B2 - sqrt(B2 * B2 - 8.0 * (double)item)) * 0.5);
        if (jj < 0) jj = 0;
        if (jj > nb - 1) jj = nb - 1;
        while (jj > 0 && (int64_t)jj * nb - (int64_t)jj * (jj - 1) / 2 > item) --jj;
        while (jj + 1 < nb && (int64_t)(jj + 1) * nb - (int64_t)(jj + 1) * jj / 2 <= item) ++jj;
        const int off = (int)(item - ((int64_t)jj * nb - (int64_t)jj * (jj - 1) / 2));
        const int j = a.fwd ? jj : nb - 1 - jj;              // column block (source)
        const int64_t oj = (int64_t)j * TH;
        const int jn = (int)((a.n - oj) < TH ? (a.n - oj) : TH);

        if (off == 0) {
            // ---- diagonal item: X_j = inv(op(T)_jj) B_j ----
            // inverse first (independent of the dependency)
            const double *D = a.dinv + (int64_t)j * TH * TH;
            for (int idx = tid; idx < TH * TH; idx += 128) {
                const int k = idx / TH, m = idx % TH;   // As[k][m] = inv(op T_jj)[m][k]
                As[k * TLD + m] = a.tT ? D[k + TH * m] : D[m + TH * k];
            }
            if (tid == 0) {
                s_ok = wait_geq(&a.cnt[j], jj, a.wait_ns, a.st);
                if (!s_ok) { atomicCAS(&a.st->timeout, 0, 1); a.st->timeout_item = (int)item; }
            }
            __syncthreads();
            if (!s_ok) return;
            for (int64_t r0 = 0; r0 < a.nrhs; r0 += NRC) {
                const int nr = (int)((a.nrhs - r0) < NRC ? (a.nrhs - r0) : NRC);
                for (int idx = tid; idx < TH * NRC; idx += 128) {
                    const int cc = idx / TH, k = idx % TH;   // Bs[k][cc] = B[oj+k, r0+cc]
                    double v = 0.0;
                    if (k < jn && cc < nr) v = __ldcg(&a.B[(oj + k) + (r0 + cc) * a.ldb]);
                    Bs[k * TLD + cc] = v;
                }
                __syncthreads();
                double acc[NRC / 8][4];
                tile_mma(As, Bs, acc, w, g, t, (nr + 7) / 8);
#pragma unroll
                for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int m = w * 16 + g + ((q & 2) ? 8 : 0);
                        const int cc = ni * 8 + 2 * t + (q & 1);
                        if (m < jn && cc < nr) a.B[(oj + m) + (r0 + cc) * a.ldb] = acc[ni][q];
                    }
                __syncthreads();
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(&a.ready[j], 1);
        } else {
            // ---- update item: B_i -= op(T)_ij X_j ----
            const int ii = jj + off;
            const int i = a.fwd ? ii : nb - 1 - ii;              // target block
            const int64_t oi = (int64_t)i * TH;
            const int in_ = (int)((a.n - oi) < TH ? (a.n - oi) : TH);
            // stage op(T)_ij (rows of block i, cols of block j) as As[k][m] = op(T)[oi+m][oj+k]
            if (!a.tT) {
                for (int idx = tid; idx < TH * TH; idx += 128) {
                    const int k = idx / TH, m = idx % TH;
                    double v = 0.0;
                    if (m < in_ && k < jn) v = (double)a.T[(oi + m) + (oj + k) * a.ldt];
                    As[k * TLD + m] = v;
                }
            } else {
                for (int idx = tid; idx < TH * TH; idx += 128) {
                    const int m = idx / TH, k = idx % TH;  // op(T)[oi+m][oj+k] = T[oj+k][oi+m]
                    double v = 0.0;
                    if (m < in_ && k < jn) v = (double)a.T[(oj + k) + (oi + m) * a.ldt];
                    As[k * TLD + m] = v;
                }
            }
            if (tid == 0) {
                s_ok = wait_geq(&a.ready[j], 1, a.wait_ns, a.st);
                if (!s_ok) { atomicCAS(&a.st->timeout, 0, 2); a.st->timeout_item = (int)item; }
            }
            __syncthreads();
            if (!s_ok) return;
            for (int64_t r0 = 0; r0 < a.nrhs; r0 += NRC) {
                const int nr = (int)((a.nrhs - r0) < NRC ? (a.nrhs - r0) : NRC);
                for (int idx = tid; idx < TH * NRC; idx += 128) {
                    const int cc = idx / TH, k = idx % TH;
                    double v = 0.0;
                    if (k < jn && cc < nr) v = __ldcg(&a.B[(oj + k) + (r0 + cc) * a.ldb]);
                    Bs[k * TLD + cc] = v;
                }
                __syncthreads();
                double acc[NRC / 8][4];
                tile_mma(As, Bs, acc, w, g, t, (nr + 7) / 8);
#pragma unroll
                for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int m = w * 16 + g + ((q & 2) ? 8 : 0);
                        const int cc = ni * 8 + 2 * t + (q & 1);
                        if (m < in_ && cc < nr) atomicAdd(&a.B[(oi + m) + (r0 + cc) * a.ldb], -acc[ni][q]);
                    }
                __syncthreads();
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) atomicAdd(&a.cnt[i], 1);
        }
    }
}

__global__ void k_scale_f64(double *B, int64_t ldb, int64_t n, int64_t nrhs, double alpha)
{
    const int64_t c = blockIdx.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        B[r + c * ldb] *= alpha;
}

}  // namespace lnb

using namespace lnb;

extern "C" int64_t lnb_trsm_sync_ints(int64_t n, int h)
{
    const int64_t nb = (n + h - 1) / h;
    return 4 + 2 * nb;
}

template <typename TT>
static int trtri_blocks(const TT *T, int64_t ldt, int64_t n, int h, char uplo, int unit, double *dinv, lnb_stream_t s)
{
    if (h != TH) return (int)cudaErrorInvalidValue;
    if (n <= 0) return 0;
    const int64_t nb = (n + TH - 1) / TH;
    const int smem = 2 * TH * (TH + 1) * (int)sizeof(double);
    cudaFuncSetAttribute(k_trtri_blocks<TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_trtri_blocks<TT><<<(unsigned)nb, TH, smem, s>>>(T, ldt, n, uplo, unit, dinv);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

template <typename TT>
static int trsm_left(char uplo, char trans, int64_t n, int64_t nrhs, double alpha, const TT *T, int64_t ldt,
                     const double *dinv, int h, double *B, int64_t ldb, int *sync, lnb_status_t *st,
                     long long wait_ns, int ticket0, lnb_stream_t s)
{
    if (h != TH) return (int)cudaErrorInvalidValue;
    if (n <= 0 || nrhs <= 0) return 0;
    cudaError_t e;
    if (alpha != 1.0) {
        dim3 grid((unsigned)((n + 255) / 256 < 128 ? (n + 255) / 256 : 128), (unsigned)nrhs);
        k_scale_f64<<<grid, 256, 0, s>>>(B, ldb, n, nrhs, alpha);
        lnb_prof_count(1);
    }
    const int64_t nsync = lnb_trsm_sync_ints(n, h);
    e = cudaMemsetAsync(sync, 0, sizeof(int) * nsync, s);
    if (e != cudaSuccess) return (int)e;
    if (ticket0 != 0) {
        e = cudaMemsetAsync(sync, ticket0 & 0xff, 1, s);  // ticket starts past item 0
        if (e != cudaSuccess) return (int)e;
    }
    TrsmArgs<TT> a;
    a.T = T; a.ldt = ldt; a.dinv = dinv; a.B = B; a.ldb = ldb; a.n = n; a.nrhs = nrhs;
    a.nb = (int)((n + TH - 1) / TH);
    const bool lowerop = (uplo == 'L') == (trans == 'N');
    a.fwd = lowerop ? 1 : 0;
    a.tT = (trans == 'T') ? 1 : 0;
    a.ticket = sync; a.cnt = sync + 4; a.ready = sync + 4 + a.nb;
    a.st = st; a.wait_ns = wait_ns;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t items = (int64_t)a.nb * (a.nb + 1) / 2;
    int64_t grid = (int64_t)sms * 4;
    if (grid > items) grid = items;
    const int smem = 2 * TH * TLD * (int)sizeof(double);
    cudaFuncSetAttribute(k_trsm_dag<TT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_trsm_dag<TT><<<(unsigned)grid, 128, smem, s>>>(a);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_trtri_blocks_f64(const double *T, int64_t ldt, int64_t n, int h, char uplo, int unit,
                                      double *dinv, lnb_stream_t s)
{
    return trtri_blocks<double>(T, ldt, n, h, uplo, unit, dinv, s);
}
extern "C" int lnb_k_trtri_blocks_f32(const float *T, int64_t ldt, int64_t n, int h, char uplo, int unit,
                                      double *dinv, lnb_stream_t s)
{
    return trtri_blocks<float>(T, ldt, n, h, uplo, unit, dinv, s);
}
extern "C" int lnb_k_trsm_left_f64(char uplo, char trans, int64_t n, int64_t nrhs, double alpha, const double *T,
                                   int64_t ldt, const double *dinv, int h, double *B, int64_t ldb, int *sync,
                                   lnb_status_t *st, long long wait_ns, int ticket0, lnb_stream_t s)
{
    return trsm_left<double>(uplo, trans, n, nrhs, alpha, T, ldt, dinv, h, B, ldb, sync, st, wait_ns, ticket0, s);
}
extern "C" int lnb_k_trsm_left_f32(char uplo, char trans, int64_t n, int64_t nrhs, double alpha, const float *T,
                                   int64_t ldt, const double *dinv, int h, double *B, int64_t ldb, int *sync,
                                   lnb_status_t *st, long long wait_ns, int ticket0, lnb_stream_t s)
{
    return trsm_left<float>(uplo, trans, n, nrhs, alpha, T, ldt, dinv, h, B, ldb, sync, st, wait_ns, ticket0, s);
}
