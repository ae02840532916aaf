// k_symv.cu -- FP64 residual kernels of the refinement loop (HBM-bound).
//
// The reference computes r = b - A x with bblas_dgemm over the full stored A
// (itref.c:1086,1094), reading 8 n^2 bytes.  A is symmetric, so here the
// product reads only the lower triangle (4 n^2 bytes): each stored element
// A[r,c] (r > c) contributes A[r,c] x[c] to y[r] and A[r,c] x[r] to y[c].
//
// Layout of the walk: a CTA owns a group of column strips and a segment of
// rows below the group's diagonal; thread t owns RPT rows, reads the strip
// elements of each (consecutive threads -> consecutive rows, so every column
// is read as contiguous runs), accumulates y[r] for its rows across the whole
// group and keeps per-column partials for the transposed contribution, which
// are reduced across the CTA once per strip.  Accumulation into y uses double
// atomics (summation order is not fixed).
#include "common.cuh"

namespace lnb {

constexpr int SV_THREADS = 256;

// Work item: SEG rows (from the item's diagonal down) x G strips of WS columns.
// Each thread owns RPT rows; their sums over the item's G*WS columns build up
// in shared memory (one atomic per row per item), and the column sums of the
// current strip build up in registers over the thread's rows (one CTA
// reduction + WS atomics per strip).  At ~128 registers two CTAs fit per SM
// and the loads of two rows per thread are in flight at once.
template <int NR>
struct SvCfg {
    static constexpr int WS = NR >= 8 ? 2 : 16 / NR;
    // 64 columns per item for every NR: the row sums take one atomic per row
    // per 64 columns (with 8 columns, the atomics of 8 right-hand sides
    // outnumbered the matrix elements and bounded the kernel)
    static constexpr int G = 64 / WS;
    static constexpr int IW = WS * G;
    static constexpr int RPT = NR >= 8 ? 2 : NR >= 4 ? 4 : 8;
    static constexpr int SEG = SV_THREADS * RPT;
};

template <int NR>
__global__ void __launch_bounds__(SV_THREADS, 2) k_symv_lower(int64_t n, const double *__restrict__ A, int64_t lda,
                                                              const double *__restrict__ X, double *Y, int absval)
{
    using Cf = SvCfg<NR>;
    constexpr int WS = Cf::WS, IW = Cf::IW, RPT = Cf::RPT;
    __shared__ double xs[IW][NR];
    __shared__ double red[SV_THREADS / 32][WS * NR];
    __shared__ double v1s[RPT * NR][SV_THREADS];     // row sums, each thread its own column
    const int64_t cj = (int64_t)blockIdx.y * IW;
    const int64_t r0 = cj + (int64_t)blockIdx.x * Cf::SEG;
    if (cj >= n || r0 >= n) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wcols = (int)((n - cj) < IW ? (n - cj) : IW);
    for (int i = tid; i < IW * NR; i += SV_THREADS) {
        const int c = i / NR, q = i % NR;
        xs[c][q] = (c < wcols) ? X[(cj + c) + (int64_t)q * n] : 0.0;
    }
    for (int i = 0; i < RPT * NR; ++i) v1s[i][tid] = 0.0;
    __syncthreads();
#pragma unroll 1
    for (int g = 0; g < Cf::G; ++g) {
        const int64_t cg = cj + g * WS;
        const int wg = wcols - g * WS;               // valid columns of this strip (may be <= 0)
        double v2[WS][NR];
#pragma unroll
        for (int c = 0; c < WS; ++c)
#pragma unroll
            for (int q = 0; q < NR; ++q) v2[c][q] = 0.0;
#pragma unroll 2
        for (int i = 0; i < RPT; ++i) {
            const int64_t r = r0 + tid + (int64_t)SV_THREADS * i;
            const double *arow = A + r + cg * lda;
            double av[WS], xr[NR], s1[NR];
#pragma unroll
            for (int c = 0; c < WS; ++c)
                av[c] = (r < n && c < wg && r >= cg + c) ? __ldcs(arow + (int64_t)c * lda) : 0.0;
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                xr[q] = r < n ? __ldg(X + r + (int64_t)q * n) : 0.0;
                s1[q] = 0.0;
            }
#pragma unroll
            for (int c = 0; c < WS; ++c) {
                const double v = absval ? fabs(av[c]) : av[c];
                const bool strict = r > cg + c;
#pragma unroll
                for (int q = 0; q < NR; ++q) {
                    s1[q] = fma(v, xs[g * WS + c][q], s1[q]);
                    if (strict) v2[c][q] = fma(v, xr[q], v2[c][q]);
                }
            }
#pragma unroll
            for (int q = 0; q < NR; ++q) v1s[i * NR + q][tid] += s1[q];
        }
        // column sums of the strip over the CTA's rows
#pragma unroll
        for (int c = 0; c < WS; ++c)
#pragma unroll
            for (int q = 0; q < NR; ++q) {
                double v = v2[c][q];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) red[warp][c * NR + q] = v;
            }
        __syncthreads();
        for (int i = tid; i < WS * NR; i += SV_THREADS) {
            double v = 0.0;
            for (int w = 0; w < SV_THREADS / 32; ++w) v += red[w][i];
            const int c = i / NR, q = i % NR;
            if (c < wg && v != 0.0) atomicAdd(&Y[(cg + c) + (int64_t)q * n], v);
        }
        __syncthreads();
    }
    for (int i = 0; i < RPT; ++i) {
        const int64_t r = r0 + tid + (int64_t)SV_THREADS * i;
        if (r < n)
            for (int q = 0; q < NR; ++q) atomicAdd(&Y[r + (int64_t)q * n], v1s[i * NR + q][tid]);
    }
}

LNB_DEV void atomic_max_nonneg(double *addr, double v)
{
    // non-negative doubles order like their bit patterns as signed 64-bit ints
    atomicMax(reinterpret_cast<long long *>(addr), __double_as_longlong(v));
}

__global__ void k_resid(int64_t n, int64_t nrhs, const double *B, int64_t ldb, const double *Y, double *R,
                        double *rmax)
{
    const int64_t q = blockIdx.y;
    double m = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const double v = B[r + q * ldb] - Y[r + q * n];
        R[r + q * n] = v;
        m = fmax(m, fabs(v));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&rmax[q], m);
}

__global__ void k_colmax(int64_t n, const double *X, int64_t ldx, double *out)
{
    const int64_t q = blockIdx.y;
    double m = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(X[r + q * ldx]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&out[q], m);
}

__global__ void k_scale_rows(int64_t n, const double *sc, const double *R, double *Z)
{
    const int64_t q = blockIdx.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        Z[r + q * n] = sc ? sc[r] * R[r + q * n] : R[r + q * n];
}

__global__ void k_axpy_scaled(int64_t n, const double *sc, const double *Z, double *X, int64_t ldx)
{
    const int64_t q = blockIdx.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        X[r + q * ldx] += (sc ? sc[r] : 1.0) * Z[r + q * n];
}

// per-column dot products out[q] = <U_q, V_q> (ld n)
__global__ void k_coldot(int64_t n, const double *U, const double *V, double *out)
{
    const int64_t q = blockIdx.y;
    double sum = 0.0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        sum = fma(U[r + q * n], V[r + q * n], sum);
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&out[q], sum);
}

// PCG step: a = num[q]/den[q];  X += a P;  R -= a Q
__global__ void k_pcg_xr(int64_t n, const double *num, const double *den, const double *P, const double *Q,
                         double *X, int64_t ldx, double *R)
{
    const int64_t q = blockIdx.y;
    const double a = num[q] / den[q];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        X[r + q * ldx] += a * P[r + q * n];
        R[r + q * n] -= a * Q[r + q * n];
    }
}

// P = Z + (num[q]/den[q]) P
__global__ void k_pcg_p(int64_t n, const double *num, const double *den, const double *Z, double *P)
{
    const int64_t q = blockIdx.y;
    const double b = num[q] / den[q];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        P[r + q * n] = Z[r + q * n] + b * P[r + q * n];
}

}  // namespace lnb

using namespace lnb;

template <int NR>
static void launch_symv(int64_t n, const double *A, int64_t lda, const double *X, double *Y, int absval,
                        lnb_stream_t s)
{
    using Cf = SvCfg<NR>;
    dim3 grid((unsigned)((n + Cf::SEG - 1) / Cf::SEG), (unsigned)((n + Cf::IW - 1) / Cf::IW));
    k_symv_lower<NR><<<grid, SV_THREADS, 0, s>>>(n, A, lda, X, Y, absval);
    lnb_prof_count(1);
}

// nrhs columns are processed in passes of 8 / 4 / 2 / 1 (X, Y with ld n)
extern "C" int lnb_k_symv_lower_f64(int64_t n, int64_t nrhs, const double *A, int64_t lda, const double *X,
                                    double *Y, int absval, lnb_stream_t s)
{
    if (n <= 0 || nrhs <= 0) return 0;
    cudaError_t e = cudaMemsetAsync(Y, 0, sizeof(double) * n * nrhs, s);
    if (e != cudaSuccess) return (int)e;
    int64_t q = 0;
    while (q < nrhs) {
        const int64_t left = nrhs - q;
        const double *Xq = X + q * n;
        double *Yq = Y + q * n;
        if (left >= 8) { launch_symv<8>(n, A, lda, Xq, Yq, absval, s); q += 8; }
        else if (left >= 4) { launch_symv<4>(n, A, lda, Xq, Yq, absval, s); q += 4; }
        else if (left >= 2) { launch_symv<2>(n, A, lda, Xq, Yq, absval, s); q += 2; }
        else { launch_symv<1>(n, A, lda, Xq, Yq, absval, s); q += 1; }
    }
    return (int)cudaGetLastError();
}

static dim3 vgrid(int64_t n, int64_t nrhs)
{
    int64_t bx = (n + 255) / 256;
    if (bx > 512) bx = 512;
    return dim3((unsigned)bx, (unsigned)nrhs);
}

extern "C" int lnb_k_resid_f64(int64_t n, int64_t nrhs, const double *B, int64_t ldb, const double *Y, double *R,
                               double *rmax, lnb_stream_t s)
{
    cudaError_t e = cudaMemsetAsync(rmax, 0, sizeof(double) * nrhs, s);
    if (e != cudaSuccess) return (int)e;
    k_resid<<<vgrid(n, nrhs), 256, 0, s>>>(n, nrhs, B, ldb, Y, R, rmax);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_colmax_f64(int64_t n, int64_t nrhs, const double *X, int64_t ldx, double *out, lnb_stream_t s)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * nrhs, s);
    if (e != cudaSuccess) return (int)e;
    k_colmax<<<vgrid(n, nrhs), 256, 0, s>>>(n, X, ldx, out);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_scale_rows_f64(int64_t n, int64_t nrhs, const double *sc, const double *R, double *Z,
                                    lnb_stream_t s)
{
    k_scale_rows<<<vgrid(n, nrhs), 256, 0, s>>>(n, sc, R, Z);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_axpy_scaled_f64(int64_t n, int64_t nrhs, const double *sc, const double *Z, double *X,
                                     int64_t ldx, lnb_stream_t s)
{
    k_axpy_scaled<<<vgrid(n, nrhs), 256, 0, s>>>(n, sc, Z, X, ldx);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_coldot_f64(int64_t n, int64_t nrhs, const double *U, const double *V, double *out,
                                lnb_stream_t s)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * nrhs, s);
    if (e != cudaSuccess) return (int)e;
    k_coldot<<<vgrid(n, nrhs), 256, 0, s>>>(n, U, V, out);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_pcg_xr_f64(int64_t n, int64_t nrhs, const double *num, const double *den, const double *P,
                                const double *Q, double *X, int64_t ldx, double *R, lnb_stream_t s)
{
    k_pcg_xr<<<vgrid(n, nrhs), 256, 0, s>>>(n, num, den, P, Q, X, ldx, R);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_pcg_p_f64(int64_t n, int64_t nrhs, const double *num, const double *den, const double *Z,
                               double *P, lnb_stream_t s)
{
    k_pcg_p<<<vgrid(n, nrhs), 256, 0, s>>>(n, num, den, Z, P);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
