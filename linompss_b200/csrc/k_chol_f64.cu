// k_chol_f64.cu -- FP64 tile kernels of the right-looking tile Cholesky.
//
//  K1 potrf   : one diagonal tile, one CTA, shared-memory staged column panels
//               (semantics of task_dpotrf -> LAPACK dpotrf 'L',
//               tasks_potrf.c:20-24; info is reported, not dropped)
//  K2 trsm    : panel solve B <- B L^-T (task_dtrsm(R,L,T,N), chol_rlmain.c:35-38)
//               on DMMA, left-looking over 32-column blocks, multiplying by the
//               inverted 32x32 diagonal blocks produced by K1
//  K3/K4 syrk : trailing update C -= P P^T restricted to r >= c: all SYRK
//               (chol_rlmain.c:48) and GEMM (chol_rlmain.c:42-46) tasks of one
//               k-step fused into one launch, 128x128 CTA tiles on DMMA with a
//               4-stage cp.async pipeline
#include "common.cuh"

#include <math.h>

namespace lnb {

// ========================================================================
// K1: diagonal tile factorization
// ========================================================================
// The tile (bs x bs, column-major, ld lda) stays in global memory (it is
// L2-resident); each NB-wide column panel is staged in shared memory,
// factored column by column, written back, and applied to the rest of the
// tile as a register-blocked (8x8 per thread) rank-NB update of the lower
// triangle.
template <int NB>
__global__ void __launch_bounds__(256) k_potrf_f64(double *A, int64_t lda, int bs, int64_t row0,
                                                   double *dinv, lnb_status_t *st)
{
    extern __shared__ double sm[];
    constexpr int LDP = NB + 1;  // panel row stride (odd: spreads banks)
    double *Pn = sm;             // [bs][LDP], row r = tile row j0 + r
    __shared__ int fail, fail_col;   // fail_col: tile-relative column of the bad pivot
    const int tid = threadIdx.x;
    if (tid == 0) { fail = 0; fail_col = bs; }

    for (int j0 = 0; j0 < bs; j0 += NB) {
        const int jb = min(NB, bs - j0);
        const int mr = bs - j0;
        __syncthreads();
        // (a) stage panel: rows j0..bs, cols j0..j0+jb
        for (int idx = tid; idx < mr * jb; idx += blockDim.x) {
            int c = idx / mr, r = idx - c * mr;
            Pn[r * LDP + c] = A[(int64_t)(j0 + r) + (int64_t)(j0 + c) * lda];
        }
        __syncthreads();
        // (b) factor the panel column by column
        for (int c = 0; c < jb; ++c) {
            if (tid == 0) {
                double d = Pn[c * LDP + c];
                if (!(d > 0.0)) {
                    fail = 1;
                    fail_col = j0 + c;
                    atomicCAS(&st->info, 0, (int)(row0 + j0 + c + 1));
                } else {
                    Pn[c * LDP + c] = sqrt(d);
                }
            }
            __syncthreads();
            if (fail) break;
            const double dc = Pn[c * LDP + c];
            for (int r = c + 1 + tid; r < mr; r += blockDim.x) Pn[r * LDP + c] /= dc;
            __syncthreads();
            const int w = jb - c - 1;
            if (w > 0) {
                const int rows = mr - c - 1;
                for (int idx = tid; idx < rows * w; idx += blockDim.x) {
                    int r = c + 1 + idx / w, cc = c + 1 + idx % w;
                    if (r >= cc) Pn[r * LDP + cc] -= Pn[r * LDP + c] * Pn[cc * LDP + c];
                }
            }
            __syncthreads();
        }
        // (c) write the factored panel back (lower part only)
        for (int idx = tid; idx < mr * jb; idx += blockDim.x) {
            int c = idx / mr, r = idx - c * mr;
            if (r >= c) A[(int64_t)(j0 + r) + (int64_t)(j0 + c) * lda] = Pn[r * LDP + c];
        }
        if (fail) break;
        // (e) rank-jb update of the trailing lower triangle of the tile
        const int tr = mr - jb;
        if (tr > 0) {
            const int nb8 = (tr + 7) / 8;
            const int nblk = nb8 * (nb8 + 1) / 2;
            for (int id = tid; id < nblk; id += blockDim.x) {
                int bi = (int)((sqrtf(8.0f * id + 1.0f) - 1.0f) * 0.5f);
                while (bi * (bi + 1) / 2 > id) --bi;
                while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
                const int bj = id - bi * (bi + 1) / 2;
                double acc[8][8];
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
                const int ra = jb + bi * 8, rb = jb + bj * 8;
                for (int p = 0; p < jb; ++p) {
                    double a[8], b[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        a[i] = (ra + i < mr) ? Pn[(ra + i) * LDP + p] : 0.0;
                        b[i] = (rb + i < mr) ? Pn[(rb + i) * LDP + p] : 0.0;
                    }
#pragma unroll
                    for (int i = 0; i < 8; ++i)
#pragma unroll
                        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int c = rb + j;
                    if (c >= mr) continue;
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int r = ra + i;
                        if (r < mr && r >= c) A[(int64_t)(j0 + r) + (int64_t)(j0 + c) * lda] -= acc[i][j];
                    }
                }
            }
        }
    }
    // (d) inverses of the 32x32 diagonal blocks of the factored tile, read
    // back from global memory (one warp per block, one lane per column).
    // After a failed pivot only the columns before it are factored: the
    // inverses treat the rest as identity, so a panel solve that follows
    // still produces exact values in those leading columns (as LAPACK's
    // partial factor does).
    if (dinv != nullptr) {
        __threadfence_block();
        __syncthreads();
        const int lane = tid & 31, warp = tid >> 5;
        const int nq = (bs + 31) / 32;
        const int lim = fail_col;
        for (int q = warp; q < nq; q += blockDim.x / 32) {
            const int qn = max(0, min(32, lim - q * 32));
            const double *Lq = A + (int64_t)q * 32 * (lda + 1);
            double *D = dinv + (int64_t)q * 1024;
            const int c = lane;
            for (int r = 0; r < 32; ++r) {
                double v;
                if (c >= qn) v = (r == c) ? 1.0 : 0.0;       // identity padding
                else if (r < c || r >= qn) v = 0.0;
                else if (r == c) v = 1.0 / Lq[(int64_t)c * (lda + 1)];
                else {
                    double s = 0.0;
                    for (int p = c; p < r; ++p) s += Lq[r + (int64_t)p * lda] * D[p + 32 * c];
                    v = -s / Lq[(int64_t)r * (lda + 1)];
                }
                D[r + 32 * c] = v;
            }
        }
    }
}

// ========================================================================
// DMMA building blocks
// ========================================================================
// Shared tiles are stored k-major: S[k][m] with a row stride of M + 4
// doubles, which spreads a half-warp's (g, t) fragment reads over all 32
// banks (stride = 4 mod 16 doubles).

// ========================================================================
// K3/K4: fused trailing update of one k-step, lower triangle only
// ========================================================================
namespace syrk {
constexpr int BM = 128, BN = 128, BK = 16, ST = 4, LDS = BM + 4;
constexpr int SMEM = 2 * ST * BK * LDS * (int)sizeof(double);
}

template <bool VEC16>
__global__ void __launch_bounds__(256) k_syrk_lower_f64(const double *__restrict__ P, int64_t ldp,
                                                        double *C, int64_t ldc, int64_t nrows,
                                                        int64_t c0, int64_t c1, int kdim)
{
    using namespace syrk;
    const int tj = blockIdx.x, ti = blockIdx.y;
    if (ti < tj) return;
    const int64_t rbase = c0 + (int64_t)ti * BM, cbase = c0 + (int64_t)tj * BN;
    if (rbase >= nrows || cbase >= c1) return;

    extern __shared__ double sm[];
    double *As = sm;                     // [ST][BK][LDS]
    double *Bs = sm + ST * BK * LDS;     // [ST][BK][LDS]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, warp tile 64 x 32
    const int g = lane >> 2, t = lane & 3;

    const int ktiles = (kdim + BK - 1) / BK;

    auto load_stage = [&](int stage, int kt) {
        const int k0 = kt * BK;
        double *as = As + stage * BK * LDS, *bs = Bs + stage * BK * LDS;
        if (VEC16) {
#pragma unroll
            for (int it = 0; it < (BK * BM / 2) / 256; ++it) {
                const int idx = tid + it * 256;
                const int kk = idx / (BM / 2), m2 = (idx % (BM / 2)) * 2;
                const bool kin = (k0 + kk) < kdim;
                const double *colp = P + (int64_t)(kin ? k0 + kk : 0) * ldp;
                {
                    const int64_t r = rbase + m2;
                    if (r + 1 < nrows) cp_async16(&as[kk * LDS + m2], colp + r, kin);
                    else {
                        const bool ok = kin && r < nrows;
                        cp_async8(&as[kk * LDS + m2], colp + (ok ? r : 0), ok);
                        cp_async8(&as[kk * LDS + m2 + 1], colp, false);
                    }
                }
                {
                    const int64_t r = cbase + m2;
                    if (r + 1 < nrows) cp_async16(&bs[kk * LDS + m2], colp + r, kin);
                    else {
                        const bool ok = kin && r < nrows;
                        cp_async8(&bs[kk * LDS + m2], colp + (ok ? r : 0), ok);
                        cp_async8(&bs[kk * LDS + m2 + 1], colp, false);
                    }
                }
            }
        } else {
#pragma unroll
            for (int it = 0; it < (BK * BM) / 256; ++it) {
                const int idx = tid + it * 256;
                const int kk = idx / BM, m = idx % BM;
                const bool kin = (k0 + kk) < kdim;
                const double *colp = P + (int64_t)(kin ? k0 + kk : 0) * ldp;
                const int64_t ra = rbase + m, rb = cbase + m;
                cp_async8(&as[kk * LDS + m], colp + (ra < nrows ? ra : 0), kin && ra < nrows);
                cp_async8(&bs[kk * LDS + m], colp + (rb < nrows ? rb : 0), kin && rb < nrows);
            }
        }
    };

    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

#pragma unroll
    for (int s = 0; s < ST - 1; ++s) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }

    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<ST - 2>();
        __syncthreads();
        {
            const int nk = kt + ST - 1;
            if (nk < ktiles) load_stage(nk % ST, nk);
            cp_async_commit();
        }
        const double *as = As + (kt % ST) * BK * LDS;
        const double *bs = Bs + (kt % ST) * BK * LDS;
#pragma unroll
        for (int kq = 0; kq < BK / 4; ++kq) {
            const double *ak = as + (kq * 4 + t) * LDS;
            const double *bk = bs + (kq * 4 + t) * LDS;
            double a0[4], a1[4], b0[4];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                a0[mi] = ak[wm * 64 + mi * 16 + g];
                a1[mi] = ak[wm * 64 + mi * 16 + g + 8];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) b0[ni] = bk[wn * 32 + ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < 4; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a0[mi], a1[mi], b0[ni]);
        }
    }
    cp_async_wait<0>();

    // epilogue: C -= acc on r >= c inside [0,nrows) x [c0,c1)
#pragma unroll
    for (int mi = 0; mi < 4; ++mi) {
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t r = rbase + wm * 64 + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int64_t c = cbase + wn * 32 + ni * 8 + 2 * t + (q & 1);
                if (r < nrows && c < c1 && r >= c) C[r + c * ldc] -= acc[mi][ni][q];
            }
        }
    }
}

// ========================================================================
// K2: panel solve B <- B L^-T, left-looking over 32-column blocks
// ========================================================================
// One CTA owns 64 rows of the panel (4 warps x 16 rows).  Column block jb:
//   T  = B[:, jb] - X[:, 0:jb] * L[jb, 0:jb]^T      (DMMA, K = 32*jb, pipelined)
//   X[:, jb] = T * Dinv_jb^T                         (DMMA, K = 32)
// where X[:, 0:jb] are this CTA's own earlier results (re-read from L2).
namespace trsm {
constexpr int BM = 64, BN = 32, BK = 16, ST = 4;
constexpr int LDX = BM + 4, LDL = BN + 4;
constexpr int SMEM = (ST * BK * LDX + ST * BK * LDL + 32 * LDX + 32 * LDL) * (int)sizeof(double);
}

__global__ void __launch_bounds__(128) k_trsm_rlt_f64(const double *__restrict__ L, int64_t lda,
                                                      const double *__restrict__ dinv, double *B,
                                                      int64_t ldb, int64_t m, int bs)
{
    using namespace trsm;
    extern __shared__ double sm[];
    double *Xs = sm;                       // [ST][BK][LDX]
    double *Ls = Xs + ST * BK * LDX;       // [ST][BK][LDL]
    double *Ts = Ls + ST * BK * LDL;       // [32][LDX]  (k = column of T, m = row)
    double *Ds = Ts + 32 * LDX;            // [32][LDL]  (k, n) = Dinv(n, k)

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int64_t rbase = (int64_t)blockIdx.x * BM;
    const int nblk = (bs + 31) / 32;

    for (int jb = 0; jb < nblk; ++jb) {
        const int jc = jb * 32;
        double acc[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[ni][q] = 0.0;

        const int ktiles = jc / BK;  // K = jc (multiple of 32)
        auto load_stage = [&](int stage, int kt) {
            const int k0 = kt * BK;
            double *xs = Xs + stage * BK * LDX, *ls = Ls + stage * BK * LDL;
            // X tile: 64 rows x 16 k, element (m, k) = B[rbase+m, k0+k]
#pragma unroll
            for (int it = 0; it < (BK * BM) / 128; ++it) {
                const int idx = tid + it * 128;
                const int kk = idx / BM, mm = idx % BM;
                const int64_t r = rbase + mm;
                cp_async8(&xs[kk * LDX + mm], B + (r < m ? r : 0) + (int64_t)(k0 + kk) * ldb, r < m);
            }
            // L tile: element (n, k) = L[jc+n, k0+k]
#pragma unroll
            for (int it = 0; it < (BK * BN) / 128; ++it) {
                const int idx = tid + it * 128;
                const int kk = idx / BN, nn = idx % BN;
                const bool ok = (jc + nn) < bs;
                cp_async8(&ls[kk * LDL + nn], L + (ok ? jc + nn : 0) + (int64_t)(k0 + kk) * lda, ok);
            }
        };

#pragma unroll
        for (int s = 0; s < ST - 1; ++s) {
            if (s < ktiles) load_stage(s, s);
            cp_async_commit();
        }
        for (int kt = 0; kt < ktiles; ++kt) {
            cp_async_wait<ST - 2>();
            __syncthreads();
            {
                const int nk = kt + ST - 1;
                if (nk < ktiles) load_stage(nk % ST, nk);
                cp_async_commit();
            }
            const double *xs = Xs + (kt % ST) * BK * LDX;
            const double *ls = Ls + (kt % ST) * BK * LDL;
#pragma unroll
            for (int kq = 0; kq < BK / 4; ++kq) {
                const double a0 = xs[(kq * 4 + t) * LDX + w * 16 + g];
                const double a1 = xs[(kq * 4 + t) * LDX + w * 16 + g + 8];
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    dmma16x8x4(acc[ni], a0, a1, ls[(kq * 4 + t) * LDL + ni * 8 + g]);
            }
        }
        cp_async_wait<0>();
        __syncthreads();

        // T = B[:, jc:jc+32] - acc  -> Ts[c][r];  Dinv_jb^T -> Ds
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int rl = w * 16 + g + ((q & 2) ? 8 : 0);
                const int cl = ni * 8 + 2 * t + (q & 1);
                const int64_t r = rbase + rl;
                double v = 0.0;
                if (r < m && jc + cl < bs) v = B[r + (int64_t)(jc + cl) * ldb] - acc[ni][q];
                Ts[cl * LDX + rl] = v;
            }
        }
        {
            const double *D = dinv + (int64_t)jb * 1024;
            for (int idx = tid; idx < 1024; idx += 128) {
                const int n = idx & 31, k = idx >> 5;  // Ds[k][n] = Dinv(n, k)
                Ds[k * LDL + n] = D[n + 32 * k];
            }
        }
        __syncthreads();
        double y[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) y[ni][q] = 0.0;
#pragma unroll
        for (int kq = 0; kq < 8; ++kq) {
            const double a0 = Ts[(kq * 4 + t) * LDX + w * 16 + g];
            const double a1 = Ts[(kq * 4 + t) * LDX + w * 16 + g + 8];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma16x8x4(y[ni], a0, a1, Ds[(kq * 4 + t) * LDL + ni * 8 + g]);
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t r = rbase + w * 16 + g + ((q & 2) ? 8 : 0);
                const int cl = ni * 8 + 2 * t + (q & 1);
                if (r < m && jc + cl < bs) B[r + (int64_t)(jc + cl) * ldb] = y[ni][q];
            }
        }
        __threadfence_block();
        __syncthreads();
    }
}

// ========================================================================
// Generic FP64 GEMM for the tile-task ABI (task_dgemm / task_dsyrk)
// ========================================================================
// C = alpha op(A) op(B) + beta C, optionally restricted to a triangle of C
// (tri = 'L' or 'U').  SIMT, 64x64 tiles, 4x4 per thread.
__global__ void __launch_bounds__(256) k_gemm_f64(char ta, char tb, int64_t M, int64_t N, int64_t K,
                                                  double alpha, const double *A, int64_t lda,
                                                  const double *Bm, int64_t ldb, double beta,
                                                  double *C, int64_t ldc, char tri)
{
    __shared__ double As[16][65], Bs[16][65];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int64_t m0 = (int64_t)blockIdx.y * 64, n0 = (int64_t)blockIdx.x * 64;
    double acc[4][4] = {};
    for (int64_t k0 = 0; k0 < K; k0 += 16) {
        for (int idx = threadIdx.x; idx < 16 * 64; idx += 256) {
            const int kk = idx / 64, mm = idx % 64;
            const int64_t k = k0 + kk, i = m0 + mm, j = n0 + mm;
            double av = 0.0, bv = 0.0;
            if (k < K && i < M) av = (ta == 'N') ? A[i + k * lda] : A[k + i * lda];
            if (k < K && j < N) bv = (tb == 'N') ? Bm[k + j * ldb] : Bm[j + k * ldb];
            As[kk][mm] = av;
            Bs[kk][mm] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = As[kk][ty + 16 * i]; b[i] = Bs[kk][tx + 16 * i]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t r = m0 + ty + 16 * i, c = n0 + tx + 16 * j;
            if (r >= M || c >= N) continue;
            if (tri == 'L' && r < c) continue;
            if (tri == 'U' && r > c) continue;
            double *cp = &C[r + c * ldc];
            *cp = (beta == 0.0 ? 0.0 : beta * *cp) + alpha * acc[i][j];
        }
}

__global__ void k_copy_lower_f64(const double *src, int64_t lds, double *dst, int64_t ldd, int64_t n)
{
    const int64_t c = blockIdx.y;
    for (int64_t r = c + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x)
        dst[r + c * ldd] = src[r + c * lds];
}

}  // namespace lnb

// ========================================================================
// launchers
// ========================================================================
using namespace lnb;

extern "C" int lnb_k_potrf_f64(double *A, int64_t lda, int bs, int64_t row0, double *dinv,
                               lnb_status_t *st, lnb_stream_t s)
{
    if (bs <= 0) return 0;
    if (bs <= 512) {
        const int smem = bs * 33 * (int)sizeof(double);
        cudaFuncSetAttribute(k_potrf_f64<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_potrf_f64<32><<<1, 256, smem, s>>>(A, lda, bs, row0, dinv, st);
        lnb_prof_count(1);
    } else if (bs <= 1024) {
        const int smem = bs * 17 * (int)sizeof(double);
        cudaFuncSetAttribute(k_potrf_f64<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        k_potrf_f64<16><<<1, 256, smem, s>>>(A, lda, bs, row0, dinv, st);
        lnb_prof_count(1);
    } else {
        return (int)cudaErrorInvalidValue;
    }
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_trsm_rlt_f64(const double *L, int64_t lda, const double *dinv, double *B,
                                  int64_t ldb, int64_t m, int bs, lnb_stream_t s)
{
    if (m <= 0 || bs <= 0) return 0;
    cudaFuncSetAttribute(k_trsm_rlt_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, trsm::SMEM);
    const int64_t grid = (m + trsm::BM - 1) / trsm::BM;
    k_trsm_rlt_f64<<<(unsigned)grid, 128, trsm::SMEM, s>>>(L, lda, dinv, B, ldb, m, bs);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_syrk_lower_f64(const double *P, int64_t ldp, double *C, int64_t ldc,
                                    int64_t nrows, int64_t c0, int64_t c1, int kdim, lnb_stream_t s)
{
    if (nrows <= c0 || c1 <= c0 || kdim <= 0) return 0;
    const int64_t tiles_c = (c1 - c0 + syrk::BN - 1) / syrk::BN;
    const int64_t tiles_r = (nrows - c0 + syrk::BM - 1) / syrk::BM;
    dim3 grid((unsigned)tiles_c, (unsigned)tiles_r);
    const bool vec = ((uintptr_t)P % 16 == 0) && (ldp % 2 == 0) && (c0 % 2 == 0);
    if (vec) {
        cudaFuncSetAttribute(k_syrk_lower_f64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, syrk::SMEM);
        k_syrk_lower_f64<true><<<grid, 256, syrk::SMEM, s>>>(P, ldp, C, ldc, nrows, c0, c1, kdim);
        lnb_prof_count(1);
    } else {
        cudaFuncSetAttribute(k_syrk_lower_f64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, syrk::SMEM);
        k_syrk_lower_f64<false><<<grid, 256, syrk::SMEM, s>>>(P, ldp, C, ldc, nrows, c0, c1, kdim);
        lnb_prof_count(1);
    }
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_gemm_f64(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                              const double *A, int64_t lda, const double *B, int64_t ldb, double beta,
                              double *C, int64_t ldc, lnb_stream_t s)
{
    return lnb_k_gemm_tri_f64(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, 0, s);
}

extern "C" int lnb_k_gemm_tri_f64(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                                  const double *A, int64_t lda, const double *B, int64_t ldb,
                                  double beta, double *C, int64_t ldc, char tri, lnb_stream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    dim3 grid((unsigned)((n + 63) / 64), (unsigned)((m + 63) / 64));
    k_gemm_f64<<<grid, 256, 0, s>>>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_copy_lower_f64(const double *src, int64_t lds, double *dst, int64_t ldd,
                                    int64_t n, lnb_stream_t s)
{
    if (n <= 0) return 0;
    dim3 grid((unsigned)((n + 255) / 256 < 64 ? (n + 255) / 256 : 64), (unsigned)n);
    k_copy_lower_f64<<<grid, 256, 0, s>>>(src, lds, dst, ldd, n);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
