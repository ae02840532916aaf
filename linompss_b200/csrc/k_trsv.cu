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
// the inverses are computed in FP64 and stored in the precision of T
template <typename TT>
__global__ void __launch_bounds__(TH) k_trtri_blocks(const TT *T, int64_t ldt, int64_t n, char uplo, int unit,
                                                     TT *dinv)
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
    TT *D = dinv + (int64_t)q * TH * TH;
    for (int r = 0; r < TH; ++r) D[r + TH * c] = (TT)X[r][c];
}

// ------------------------------------------------------------------------
// the DAG walk
// ------------------------------------------------------------------------
template <typename TT>
struct TrsmArgs {
    const TT *T; int64_t ldt; const TT *dinv;
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

// stage op(T)(block row oi, block col oj) as As[k][m] = op(T)[oi+m][oj+k] (zero-padded)
template <typename TT>
LNB_DEV void stage_tile(const TrsmArgs<TT> &a, double *As, int64_t oi, int in_, int64_t oj, int jn, int tid)
{
    if (!a.tT) {
        for (int idx = tid; idx < TH * TH; idx += 128) {
            const int k = idx / TH, m = idx % TH;
            As[k * TLD + m] = (m < in_ && k < jn) ? (double)a.T[(oi + m) + (oj + k) * a.ldt] : 0.0;
        }
    } else {
        for (int idx = tid; idx < TH * TH; idx += 128) {
            const int m = idx / TH, k = idx % TH;     // op(T)[oi+m][oj+k] = T[oj+k][oi+m]
            As[k * TLD + m] = (m < in_ && k < jn) ? (double)a.T[(oj + k) + (oi + m) * a.ldt] : 0.0;
        }
    }
}

// rhs rows [o, o+rows) x columns [r0, r0+nr) as Bs[k][cc] (k-major), zero-padded
LNB_DEV void stage_rhs(const double *B, int64_t ldb, double *Bs, int64_t o, int rows, int64_t r0, int nr, int tid)
{
    for (int idx = tid; idx < TH * NRC; idx += 128) {
        const int cc = idx / TH, k = idx % TH;
        Bs[k * TLD + cc] = (k < rows && cc < nr) ? __ldcg(&B[(o + k) + (r0 + cc) * ldb]) : 0.0;
    }
}

// Work items in row order of the lower block triangle (virtual rows, reversed
// for an upper op(T)): row ii holds the off-diagonal updates U(ii, jj) for
// jj <= ii-2, then the row item R(ii).  R(ii) absorbs the sub-diagonal update
// U(ii, ii-1) -- the only one on the critical chain --, so the chain per
// block is R(ii-1) -> R(ii): wait X_{ii-1}, one prefetched 64x64 tile product,
// one prefetched inverse product, publish X_ii.  Every item waits only on
// items with smaller tickets.
template <typename TT>
__global__ void __launch_bounds__(128) k_trsm_dag(TrsmArgs<TT> a)
{
    extern __shared__ double smd[];
    double *As = smd;                  // [TH][TLD] tile of op(T)
    double *Ds = smd + TH * TLD;       // [TH][TLD] inverse of the diagonal block
    double *Bs = smd + 2 * TH * TLD;   // [TH][TLD] rhs chunk
    __shared__ int s_item, s_ok;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = lane >> 2, t = lane & 3;
    const int nb = a.nb;
    const int64_t total = 1 + (int64_t)nb * (nb - 1) / 2;

    while (true) {
        if (tid == 0) s_item = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int64_t item = s_item;
        __syncthreads();
        if (item >= total) break;

        // decode: row ii >= 1 starts at 1 + (ii-1) ii / 2
        int ii = 0, off = 0;
        if (item > 0) {
            ii = (int)((1.0 + sqrt(1.0 + 8.0 * (double)(item - 1))) * 0.5);
            if (ii < 1) ii = 1;
            while (ii > 1 && 1 + (int64_t)(ii - 1) * ii / 2 > item) --ii;
            while (1 + (int64_t)ii * (ii + 1) / 2 <= item) ++ii;
            off = (int)(item - (1 + (int64_t)(ii - 1) * ii / 2));
        }
        const bool row_item = (ii == 0) || (off == ii - 1);
        const int i = a.fwd ? ii : nb - 1 - ii;
        const int64_t oi = (int64_t)i * TH;
        const int in_ = (int)((a.n - oi) < TH ? (a.n - oi) : TH);

        if (row_item) {
            // ---- R(ii): X_i = inv(op T_ii) (B_i - op(T)_{i,p} X_p),  p = previous block ----
            const TT *D = a.dinv + (int64_t)i * TH * TH;
            for (int idx = tid; idx < TH * TH; idx += 128) {
                const int k = idx / TH, m = idx % TH;   // Ds[k][m] = inv(op T_ii)[m][k]
                Ds[k * TLD + m] = a.tT ? D[k + TH * m] : D[m + TH * k];
            }
            const int p = a.fwd ? i - 1 : i + 1;
            const int64_t op_ = (int64_t)p * TH;
            const int pn = ii > 0 ? (int)((a.n - op_) < TH ? (a.n - op_) : TH) : 0;
            if (ii > 0) stage_tile(a, As, oi, in_, op_, pn, tid);
            if (tid == 0) {
                s_ok = wait_geq(&a.cnt[i], ii - 1, a.wait_ns, a.st);
                if (s_ok && ii > 0) s_ok = wait_geq(&a.ready[p], 1, a.wait_ns, a.st);
                if (!s_ok) { atomicCAS(&a.st->timeout, 0, 1); a.st->timeout_item = (int)item; }
            }
            __syncthreads();
            if (!s_ok) return;
            for (int64_t r0 = 0; r0 < a.nrhs; r0 += NRC) {
                const int nr = (int)((a.nrhs - r0) < NRC ? (a.nrhs - r0) : NRC);
                double acc[NRC / 8][4];
                if (ii > 0) {
                    stage_rhs(a.B, a.ldb, Bs, op_, pn, r0, nr, tid);      // X_p
                    __syncthreads();
                    tile_mma(As, Bs, acc, w, g, t, (nr + 7) / 8);
                    __syncthreads();
                } else {
#pragma unroll
                    for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
                        for (int q = 0; q < 4; ++q) acc[ni][q] = 0.0;
                }
                // Bs[m][cc] = B_i - acc   (m becomes k of the inverse product)
#pragma unroll
                for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int m = w * 16 + g + ((q & 2) ? 8 : 0);
                        const int cc = ni * 8 + 2 * t + (q & 1);
                        double v = 0.0;
                        if (m < in_ && cc < nr) v = __ldcg(&a.B[(oi + m) + (r0 + cc) * a.ldb]) - acc[ni][q];
                        Bs[m * TLD + cc] = v;
                    }
                __syncthreads();
                tile_mma(Ds, Bs, acc, w, g, t, (nr + 7) / 8);
#pragma unroll
                for (int ni = 0; ni < NRC / 8; ++ni)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int m = w * 16 + g + ((q & 2) ? 8 : 0);
                        const int cc = ni * 8 + 2 * t + (q & 1);
                        if (m < in_ && cc < nr) a.B[(oi + m) + (r0 + cc) * a.ldb] = acc[ni][q];
                    }
                __syncthreads();
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(&a.ready[i], 1);
        } else {
            // ---- U(ii, jj): B_i -= op(T)_ij X_j ----
            const int jj = off;
            const int j = a.fwd ? jj : nb - 1 - jj;
            const int64_t oj = (int64_t)j * TH;
            const int jn = (int)((a.n - oj) < TH ? (a.n - oj) : TH);
            stage_tile(a, As, oi, in_, oj, jn, tid);
            if (tid == 0) {
                s_ok = wait_geq(&a.ready[j], 1, a.wait_ns, a.st);
                if (!s_ok) { atomicCAS(&a.st->timeout, 0, 2); a.st->timeout_item = (int)item; }
            }
            __syncthreads();
            if (!s_ok) return;
            for (int64_t r0 = 0; r0 < a.nrhs; r0 += NRC) {
                const int nr = (int)((a.nrhs - r0) < NRC ? (a.nrhs - r0) : NRC);
                stage_rhs(a.B, a.ldb, Bs, oj, jn, r0, nr, tid);
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
static int trtri_blocks(const TT *T, int64_t ldt, int64_t n, int h, char uplo, int unit, TT *dinv, lnb_stream_t s)
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
                     const TT *dinv, int h, double *B, int64_t ldb, int *sync, lnb_status_t *st,
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
    if (nrhs <= 8) {
        if constexpr (sizeof(TT) == 8)
            return lnb_k_trsm_chain_f64(uplo, trans, n, nrhs, (const double *)T, ldt, (const double *)dinv, B, ldb,
                                        sync, st, wait_ns, s);
        else
            return lnb_k_trsm_chain_f32(uplo, trans, n, nrhs, (const float *)T, ldt, (const float *)dinv, B, ldb,
                                        sync, st, wait_ns, s);
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
    const int64_t items = 1 + (int64_t)a.nb * (a.nb - 1) / 2;
    int64_t grid = (int64_t)sms * 4;
    if (grid > items) grid = items;
    const int smem = 3 * TH * TLD * (int)sizeof(double);
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
                                      float *dinv, lnb_stream_t s)
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
                                   int64_t ldt, const float *dinv, int h, double *B, int64_t ldb, int *sync,
                                   lnb_status_t *st, long long wait_ns, int ticket0, lnb_stream_t s)
{
    return trsm_left<float>(uplo, trans, n, nrhs, alpha, T, ldt, dinv, h, B, ldb, sync, st, wait_ns, ticket0, s);
}
