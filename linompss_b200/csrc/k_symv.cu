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
#include <stdlib.h>

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

// ---- several right-hand sides on the FP64 tensor cores ---------------------
//
// With 2..8 right-hand sides each stored element costs 2 nr FMAs, as many as
// the HBM stream can feed, so both products go to DMMA (m16n8k4, N = 8 = the
// right-hand-side pass).  A work item is a 256 x 256 block of the lower
// triangle (4 x 4 tiles of 64 x 64); tiles stream through shared memory by
// cp.async, double-buffered, two CTAs per SM.  Per tile, warps 0-3 form
// y_I += T x_J (one 16-row slab each) and warps 4-7 form y_J += T^T x_I (one
// 16-column slab each).  y_I builds up in registers over the item's tile row
// and y_J over the whole item, so Y takes (4 + 4) x 64 x 8 atomic adds per 16
// tiles.  A diagonal tile holds only its lower triangle: the row warps read
// the mirrored element above the diagonal and the column warps skip it.
namespace symtc {
constexpr int TS = 64, LD = 68, RB = 4, NT = 256, STAGES = 2;
constexpr int BR = RB * TS;                       // rows of an item's block
struct Smem {
    double t[STAGES][TS * LD];
    double xi[BR * 8];                            // x rows of the item's row block, 8 per row (swizzled)
    double xj[BR * 8];                            // and of its column block
};
// element (row, q) of a staged x block; the swizzle keeps the B-fragment
// loads (rows 4kk + t, column g) free of bank conflicts
LNB_DEV int xoff(int row, int q) { return row * 8 + (q ^ (((row >> 1) & 1) << 2)); }

LNB_DEV void load_tile(double *dst, const double *A, int64_t lda, int64_t n, int64_t R, int64_t Cc, bool diag,
                       int tid)
{
#pragma unroll
    for (int k = 0; k < (TS * TS / 2) / NT; ++k) {
        const int ch = tid + k * NT;
        const int c = ch >> 5, rp = (ch & 31) * 2;
        if (diag && rp + 1 < c) continue;         // strictly above the diagonal: never read
        const int64_t gr = R + rp, gc = Cc + c;
        int bytes = 0;
        if (gc < n && gr < n) bytes = (n - gr) >= 2 ? 16 : 8;
        const double *src = bytes ? A + gr + gc * lda : A;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst + c * LD + rp)),
                     "l"(src), "r"(bytes));
    }
}

__global__ void __launch_bounds__(NT, 2) k_symv_tc(int64_t n, int64_t nB, const double *__restrict__ A, int64_t lda,
                                                   const double *__restrict__ X, int nr, double *Y)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem &S = *reinterpret_cast<Smem *>(smraw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
    // item -> (bi, bj), bi >= bj, row-major over the lower triangle of the block grid
    const int64_t idx = blockIdx.x;
    int64_t bi = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
    while (bi * (bi + 1) / 2 > idx) --bi;
    while ((bi + 1) * (bi + 2) / 2 <= idx) ++bi;
    const int64_t bj = idx - bi * (bi + 1) / 2;
    (void)nB;
    const bool diag = bi == bj;
    const int64_t r0 = bi * BR, c0 = bj * BR;
    const int nti = (int)min((int64_t)RB, (n - r0 + TS - 1) / TS);
    const int ntj = (int)min((int64_t)RB, (n - c0 + TS - 1) / TS);
    const int ntiles = diag ? nti * (nti + 1) / 2 : nti * ntj;

    auto decode = [&](int i, int &ii, int &jj) {
        if (diag) {
            ii = 0;
            while ((ii + 1) * (ii + 2) / 2 <= i) ++ii;
            jj = i - ii * (ii + 1) / 2;
        } else {
            ii = i / ntj;
            jj = i - ii * ntj;
        }
    };
    auto issue = [&](int i) {
        if (i < ntiles) {
            int ii, jj;
            decode(i, ii, jj);
            load_tile(S.t[i % STAGES], A, lda, n, r0 + ii * TS, c0 + jj * TS, diag && ii == jj, tid);
        }
        cp_async_commit();
    };
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) issue(s);

    for (int e = tid; e < BR * 8; e += NT) {
        const int q = e / BR, row = e - q * BR;
        const int64_t ri = r0 + row, rj = c0 + row;
        S.xi[xoff(row, q)] = (q < nr && ri < n) ? X[ri + (int64_t)q * n] : 0.0;
        S.xj[xoff(row, q)] = (q < nr && rj < n) ? X[rj + (int64_t)q * n] : 0.0;
    }

    const bool roww = warp < 4;
    const int m16 = (warp & 3) * 16;
    double accC[RB][4];
#pragma unroll
    for (int j = 0; j < RB; ++j)
#pragma unroll
        for (int v = 0; v < 4; ++v) accC[j][v] = 0.0;
    int tc = 0;
    for (int ii = 0; ii < nti; ++ii) {
        double accR[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int jj = 0; jj < RB; ++jj) {
            if (jj >= ntj || (diag && jj > ii)) continue;
            issue(tc + STAGES - 1);
            cp_async_wait<STAGES - 1>();
            __syncthreads();
            const double *T = S.t[tc % STAGES];
            const bool dt = diag && jj == ii;
            if (roww) {
                const double *xb = S.xj + jj * TS * 8;
                if (!dt) {
#pragma unroll
                    for (int kk = 0; kk < TS / 4; ++kk) {
                        const int c = 4 * kk + t4;
                        dmma16x8x4(accR, T[c * LD + m16 + g], T[c * LD + m16 + g + 8], xb[xoff(c, g)]);
                    }
                } else {
#pragma unroll
                    for (int kk = 0; kk < TS / 4; ++kk) {
                        const int c = 4 * kk + t4, ra = m16 + g, rb = ra + 8;
                        const double a0 = ra >= c ? T[c * LD + ra] : T[ra * LD + c];
                        const double a1 = rb >= c ? T[c * LD + rb] : T[rb * LD + c];
                        dmma16x8x4(accR, a0, a1, xb[xoff(c, g)]);
                    }
                }
            } else if (!dt) {
                const double *xb = S.xi + ii * TS * 8;
#pragma unroll
                for (int kk = 0; kk < TS / 4; ++kk) {
                    const int r = 4 * kk + t4;
                    dmma16x8x4(accC[jj], T[(m16 + g) * LD + r], T[(m16 + g + 8) * LD + r], xb[xoff(r, g)]);
                }
            }
            __syncthreads();
            ++tc;
        }
        if (roww) {
            const int64_t ra = r0 + ii * TS + m16 + g, rb = ra + 8;
            const int q0 = 2 * t4, q1 = q0 + 1;
            if (ra < n) {
                if (q0 < nr) atomicAdd(Y + ra + (int64_t)q0 * n, accR[0]);
                if (q1 < nr) atomicAdd(Y + ra + (int64_t)q1 * n, accR[1]);
            }
            if (rb < n) {
                if (q0 < nr) atomicAdd(Y + rb + (int64_t)q0 * n, accR[2]);
                if (q1 < nr) atomicAdd(Y + rb + (int64_t)q1 * n, accR[3]);
            }
        }
    }
    if (!roww) {
#pragma unroll
        for (int jj = 0; jj < RB; ++jj) {
            if (jj >= ntj || (diag && jj == nti - 1)) continue;   // the last diagonal column has no tile below
            const int64_t ca = c0 + jj * TS + m16 + g, cb = ca + 8;
            const int q0 = 2 * t4, q1 = q0 + 1;
            if (ca < n) {
                if (q0 < nr) atomicAdd(Y + ca + (int64_t)q0 * n, accC[jj][0]);
                if (q1 < nr) atomicAdd(Y + ca + (int64_t)q1 * n, accC[jj][1]);
            }
            if (cb < n) {
                if (q0 < nr) atomicAdd(Y + cb + (int64_t)q0 * n, accC[jj][2]);
                if (q1 < nr) atomicAdd(Y + cb + (int64_t)q1 * n, accC[jj][3]);
            }
        }
    }
    cp_async_wait<0>();
}
}  // namespace symtc

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

static bool symv_tc_enabled()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("LNB_SYMV_TC");      /* 0: the strip kernel for every right-hand-side count */
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v == 1;
}

// nrhs columns are processed in passes of 8 (tensor cores, 2..8 columns per
// pass) or, on the strip kernel, of 8 / 4 / 2 / 1 (X, Y with ld n)
extern "C" int lnb_k_symv_lower_f64(int64_t n, int64_t nrhs, const double *A, int64_t lda, const double *X,
                                    double *Y, int absval, lnb_stream_t s)
{
    if (n <= 0 || nrhs <= 0) return 0;
    cudaError_t e = cudaMemsetAsync(Y, 0, sizeof(double) * n * nrhs, s);
    if (e != cudaSuccess) return (int)e;
    /* the tensor-core pass stages A by 16-byte copies: A 16-byte aligned, lda even */
    const bool use_tc = !absval && symv_tc_enabled() && (lda % 2) == 0 && ((uintptr_t)A % 16) == 0;
    if (use_tc) {
        static int attr_set = 0;
        if (!attr_set) {
            e = cudaFuncSetAttribute(symtc::k_symv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(symtc::Smem));
            if (e != cudaSuccess) return (int)e;
            attr_set = 1;
        }
    }
    int64_t q = 0;
    while (q < nrhs) {
        const int64_t left = nrhs - q;
        const double *Xq = X + q * n;
        double *Yq = Y + q * n;
        if (left >= 2 && use_tc) {
            const int nr = left >= 8 ? 8 : (int)left;
            const int64_t nB = (n + symtc::BR - 1) / symtc::BR;
            symtc::k_symv_tc<<<(unsigned)(nB * (nB + 1) / 2), symtc::NT, sizeof(symtc::Smem), s>>>(n, nB, A, lda, Xq,
                                                                                                 nr, Yq);
            lnb_prof_count(1);
            q += nr;
        }
        else if (left >= 8) { launch_symv<8>(n, A, lda, Xq, Yq, absval, s); q += 8; }
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
