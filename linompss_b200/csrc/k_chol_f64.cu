// k_chol_f64.cu -- FP64 tile kernels of the right-looking tile Cholesky.
//
//  K1 potrf   : leaf diagonal tile (<= 128), one CTA, tile resident in shared
//               memory (k_potrf.cuh; task_dpotrf -> LAPACK dpotrf 'L',
//               tasks_potrf.c:20-24; info is reported, not dropped)
//  K2 trsm    : panel solve B <- B L^-T (task_dtrsm(R,L,T,N), chol_rlmain.c:35-38)
//               on DMMA, left-looking over 32-column blocks, multiplying by the
//               inverted 32x32 diagonal blocks produced by K1
//  K3/K4 syrk : trailing update C -= P P^T restricted to r >= c: all SYRK
//               (chol_rlmain.c:48) and GEMM (chol_rlmain.c:42-46) tasks of one
//               k-step fused into one launch, 128x128 CTA tiles on DMMA with a
//               4-stage cp.async pipeline
#include "common.cuh"
#include "k_potrf.cuh"

#include <math.h>
#include <stdlib.h>

namespace lnb {

// ========================================================================
// DMMA building blocks
// ========================================================================
// Shared tiles are stored k-major: S[k][m] with a row stride of M + 4
// doubles, which spreads a half-warp's (g, t) fragment reads over all 32
// banks (stride = 4 mod 16 doubles).

// ========================================================================
// K3/K4: fused trailing update of one k-step, lower triangle only
// ========================================================================
// Tile shapes are template parameters (CTA tile BM x BN, warp grid WM x WN,
// ST pipeline stages); the launcher picks one (see lnb_k_syrk_lower_f64).
template <int BM, int BN, int WM, int WN, int ST>
struct SyrkCfg {
    static constexpr int BK = 16;
    static constexpr int THREADS = 32 * WM * WN;
    static constexpr int LDA = BM + 4, LDB = BN + 4;     // k-major rows, = 4 mod 16 doubles
    static constexpr int TM = BM / WM, TN = BN / WN;    // warp tile
    static constexpr int MI = TM / 16, NI = TN / 8;     // DMMA tiles per warp
    static constexpr int SMEM = ST * BK * (LDA + LDB) * (int)sizeof(double);
};

template <class Cfg, int ST, bool VEC16>
__global__ void __launch_bounds__(Cfg::THREADS) k_syrk_lower_f64(const double *__restrict__ P, int64_t ldp,
                                                                 double *C, int64_t ldc, int64_t nrows,
                                                                 int64_t c0, int64_t c1, int kdim)
{
    constexpr int BK = Cfg::BK, LDA = Cfg::LDA, LDB = Cfg::LDB, THREADS = Cfg::THREADS;
    constexpr int BM = Cfg::LDA - 4, BN = Cfg::LDB - 4;
    constexpr int MI = Cfg::MI, NI = Cfg::NI, TM = Cfg::TM, TN = Cfg::TN;
    constexpr int WN = BN / TN;
    const int tj = blockIdx.x, ti = blockIdx.y;
    const int64_t rbase = c0 + (int64_t)ti * BM, cbase = c0 + (int64_t)tj * BN;
    if (rbase + BM <= cbase) return;               // tile entirely above the diagonal
    if (rbase >= nrows || cbase >= c1) return;

    extern __shared__ double sm[];
    double *As = sm;                     // [ST][BK][LDA]
    double *Bs = sm + ST * BK * LDA;     // [ST][BK][LDB]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp / WN, wn = warp % WN;
    const int g = lane >> 2, t = lane & 3;

    const int ktiles = (kdim + BK - 1) / BK;

    auto load_rows = [&](double *dst, int ld, int64_t base, int rows, int k0) {
        if (VEC16) {
            for (int idx = tid; idx < BK * rows / 2; idx += THREADS) {
                const int kk = idx / (rows / 2), m2 = (idx % (rows / 2)) * 2;
                const bool kin = (k0 + kk) < kdim;
                const double *colp = P + (int64_t)(kin ? k0 + kk : 0) * ldp;
                const int64_t r = base + m2;
                if (r + 1 < nrows) {
                    cp_async16(&dst[kk * ld + m2], colp + r, kin);
                } else {
                    const bool ok = kin && r < nrows;
                    cp_async8(&dst[kk * ld + m2], colp + (ok ? r : 0), ok);
                    cp_async8(&dst[kk * ld + m2 + 1], colp, false);
                }
            }
        } else {
            for (int idx = tid; idx < BK * rows; idx += THREADS) {
                const int kk = idx / rows, m = idx % rows;
                const bool kin = (k0 + kk) < kdim;
                const double *colp = P + (int64_t)(kin ? k0 + kk : 0) * ldp;
                const int64_t r = base + m;
                cp_async8(&dst[kk * ld + m], colp + (r < nrows ? r : 0), kin && r < nrows);
            }
        }
    };
    auto load_stage = [&](int stage, int kt) {
        load_rows(As + stage * BK * LDA, LDA, rbase, BM, kt * BK);
        load_rows(Bs + stage * BK * LDB, LDB, cbase, BN, kt * BK);
    };

    double acc[MI][NI][4];
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NI; ++j)
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
        const double *as = As + (kt % ST) * BK * LDA;
        const double *bs = Bs + (kt % ST) * BK * LDB;
#pragma unroll
        for (int kq = 0; kq < BK / 4; ++kq) {
            const double *ak = as + (kq * 4 + t) * LDA + wm * TM;
            const double *bk = bs + (kq * 4 + t) * LDB + wn * TN;
            double a0[MI], a1[MI], b0[NI];
#pragma unroll
            for (int mi = 0; mi < MI; ++mi) {
                a0[mi] = ak[mi * 16 + g];
                a1[mi] = ak[mi * 16 + g + 8];
            }
#pragma unroll
            for (int ni = 0; ni < NI; ++ni) b0[ni] = bk[ni * 8 + g];
#pragma unroll
            for (int mi = 0; mi < MI; ++mi)
#pragma unroll
                for (int ni = 0; ni < NI; ++ni) dmma16x8x4(acc[mi][ni], a0[mi], a1[mi], b0[ni]);
        }
    }
    cp_async_wait<0>();

    // epilogue: C -= acc on r >= c inside [0,nrows) x [c0,c1).  Per m16 row
    // block, every load is issued before any store (through one pointer the
    // compiler would otherwise serialize each read-modify-write).
#pragma unroll
    for (int mi = 0; mi < MI; ++mi) {
        double cv[NI][4];
#pragma unroll
        for (int ni = 0; ni < NI; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t r = rbase + wm * TM + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int64_t c = cbase + wn * TN + ni * 8 + 2 * t + (q & 1);
                cv[ni][q] = (r < nrows && c < c1 && r >= c) ? C[r + c * ldc] : 0.0;
            }
#pragma unroll
        for (int ni = 0; ni < NI; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t r = rbase + wm * TM + mi * 16 + g + ((q & 2) ? 8 : 0);
                const int64_t c = cbase + wn * TN + ni * 8 + 2 * t + (q & 1);
                if (r < nrows && c < c1 && r >= c) C[r + c * ldc] = cv[ni][q] - acc[mi][ni][q];
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
// FP64 GEMM of the tile-task ABI (task_dgemm / task_dsyrk / ompss_dsyrk)
// ========================================================================
// C = alpha op(A) op(B) + beta C, optionally restricted to a triangle of C
// (tri = 'L' or 'U'), on DMMA: 64 x 64 CTA tiles, 4 warps of 32 x 32, BK = 16,
// 4-stage cp.async pipeline, two CTAs per SM.  Each operand is staged in the
// orientation its memory is contiguous in, so every copy is a 16-byte
// cp.async along a column: op(A) = A and op(B) = B^T are stored k-major
// (S[k][m], row stride 68), op(A) = A^T and op(B) = B m-major (S[m][k], row
// stride 20).  Both strides spread a half-warp's fragment reads over all 32
// banks.  beta == 0 does not read C (BLAS semantics).
namespace gm {
constexpr int BM = 64, BN = 64, BK = 16, ST = 4, THREADS = 128;
constexpr int LDKM = BM + 4;                  // k-major row stride (doubles)
constexpr int LDMK = BK + 4;                  // m-major row stride
constexpr int STAGE = (BM * LDMK > BK * LDKM) ? BM * LDMK : BK * LDKM;
constexpr int SMEM = ST * 2 * STAGE * (int)sizeof(double);

// two consecutive elements src[0], src[1] (nv of them valid) -> dst[0..1]
LNB_DEV void load2(double *dst, const double *src, int nv)
{
    if (nv == 2 && ((uintptr_t)src & 15) == 0) {
        cp_async16(dst, src, true);
    } else {
        cp_async8(dst, nv > 0 ? src : dst, nv > 0);
        cp_async8(dst + 1, nv > 1 ? src + 1 : dst, nv > 1);
    }
}

// rows x BK tile of an operand whose element (r, k) is X[r + k ldx] (KM:
// contiguous in r -> k-major smem) or X[k + r ldx] (!KM: contiguous in k ->
// r-major smem); rows [r0, r0 + 64) of nr, k in [k0, k0 + BK) of nk
template <bool KM>
LNB_DEV void load_op(double *dst, const double *X, int64_t ldx, int64_t r0, int64_t nr, int64_t k0, int64_t nk,
                     int tid)
{
#pragma unroll
    for (int it = 0; it < (BM * BK / 2) / THREADS; ++it) {
        const int idx = tid + it * THREADS;
        if (KM) {
            const int kk = idx / (BM / 2), rr = (idx % (BM / 2)) * 2;
            const int64_t r = r0 + rr, k = k0 + kk;
            const int nv = k < nk ? (int)(r + 1 < nr ? 2 : (r < nr ? 1 : 0)) : 0;
            load2(dst + kk * LDKM + rr, X + (nv ? r + k * ldx : 0), nv);
        } else {
            const int rr = idx / (BK / 2), kk = (idx % (BK / 2)) * 2;
            const int64_t r = r0 + rr, k = k0 + kk;
            const int nv = r < nr ? (int)(k + 1 < nk ? 2 : (k < nk ? 1 : 0)) : 0;
            load2(dst + rr * LDMK + kk, X + (nv ? k + r * ldx : 0), nv);
        }
    }
}

// AKM: op(A) = A (k-major staging); BKM: op(B) = B^T (k-major staging)
template <bool AKM, bool BKM>
__global__ void __launch_bounds__(THREADS, 2) k_gemm_dmma(int64_t M, int64_t N, int64_t K, double alpha,
                                                          const double *__restrict__ A, int64_t lda,
                                                          const double *__restrict__ B, int64_t ldb, double beta,
                                                          double *C, int64_t ldc, char tri)
{
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    if (tri == 'L' && m0 + BM <= n0) return;
    if (tri == 'U' && n0 + BN <= m0) return;
    extern __shared__ __align__(16) double gsm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
    const int ktiles = (int)((K + BK - 1) / BK);
    auto stage = [&](int s, int kt) {
        double *as = gsm + (2 * s) * STAGE, *bs = gsm + (2 * s + 1) * STAGE;
        load_op<AKM>(as, A, lda, m0, M, (int64_t)kt * BK, K, tid);
        load_op<BKM>(bs, B, ldb, n0, N, (int64_t)kt * BK, K, tid);
    };
    double acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
#pragma unroll
    for (int s = 0; s < ST - 1; ++s) {
        if (s < ktiles) stage(s, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<ST - 2>();
        __syncthreads();
        {
            const int nk = kt + ST - 1;
            if (nk < ktiles) stage(nk % ST, nk);
            cp_async_commit();
        }
        const double *as = gsm + (2 * (kt % ST)) * STAGE, *bs = gsm + (2 * (kt % ST) + 1) * STAGE;
#pragma unroll
        for (int kq = 0; kq < BK / 4; ++kq) {
            const int k = kq * 4 + t;
            double a0[2], a1[2], b0[4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) {
                const int r = wm * 32 + mi * 16 + g;
                a0[mi] = AKM ? as[k * LDKM + r] : as[r * LDMK + k];
                a1[mi] = AKM ? as[k * LDKM + r + 8] : as[(r + 8) * LDMK + k];
            }
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int c = wn * 32 + ni * 8 + g;
                b0[ni] = BKM ? bs[k * LDKM + c] : bs[c * LDMK + k];
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a0[mi], a1[mi], b0[ni]);
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t r = m0 + wm * 32 + mi * 16 + g + (q >> 1) * 8;
                const int64_t c = n0 + wn * 32 + ni * 8 + 2 * t + (q & 1);
                if (r >= M || c >= N) continue;
                if (tri == 'L' && r < c) continue;
                if (tri == 'U' && r > c) continue;
                double *cp = &C[r + c * ldc];
                *cp = (beta == 0.0 ? 0.0 : beta * *cp) + alpha * acc[mi][ni][q];
            }
}
}  // namespace gm

}  // namespace lnb

// ========================================================================
// launchers
// ========================================================================
using namespace lnb;

extern "C" int lnb_k_potrf_f64(double *A, int64_t lda, int bs, int64_t row0, double *dinv,
                               lnb_status_t *st, lnb_stream_t s)
{
    if (bs <= 0) return 0;
    if (bs > LEAF) return (int)cudaErrorInvalidValue;
    const int smem = (int)leaf_smem_bytes<double>(bs);
    cudaFuncSetAttribute(k_potrf_leaf<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_potrf_leaf<double><<<1, 256, smem, s>>>(A, lda, bs, row0, dinv, st);
    lnb_prof_count(1);
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

template <int BM, int BN, int WM, int WN, int ST>
static int launch_syrk(const double *P, int64_t ldp, double *C, int64_t ldc, int64_t nrows, int64_t c0,
                       int64_t c1, int kdim, lnb_stream_t s)
{
    using Cfg = SyrkCfg<BM, BN, WM, WN, ST>;
    const int64_t tiles_c = (c1 - c0 + BN - 1) / BN;
    const int64_t tiles_r = (nrows - c0 + BM - 1) / BM;
    dim3 grid((unsigned)tiles_c, (unsigned)tiles_r);
    const bool vec = ((uintptr_t)P % 16 == 0) && (ldp % 2 == 0) && (c0 % 2 == 0);
    if (vec) {
        cudaFuncSetAttribute(k_syrk_lower_f64<Cfg, ST, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
        k_syrk_lower_f64<Cfg, ST, true><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(P, ldp, C, ldc, nrows, c0, c1, kdim);
    } else {
        cudaFuncSetAttribute(k_syrk_lower_f64<Cfg, ST, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
        k_syrk_lower_f64<Cfg, ST, false><<<grid, Cfg::THREADS, Cfg::SMEM, s>>>(P, ldp, C, ldc, nrows, c0, c1, kdim);
    }
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

static int g_syrk_cfg = -1;

// Tile shape of the trailing update.  0: 128x128 (8 warps, 4 stages);
// 1: 64x64 (4 warps, 4 stages); 2: 128x64 (4 warps, 3 stages).  The default
// is the measured-fastest on B200; LNB_SYRK_TILE overrides it (tuning).
extern "C" int lnb_k_syrk_lower_f64(const double *P, int64_t ldp, double *C, int64_t ldc,
                                    int64_t nrows, int64_t c0, int64_t c1, int kdim, lnb_stream_t s)
{
    if (nrows <= c0 || c1 <= c0 || kdim <= 0) return 0;
    if (g_syrk_cfg < 0) {
        const char *e = getenv("LNB_SYRK_TILE");
        g_syrk_cfg = e ? atoi(e) : 1;
    }
    switch (g_syrk_cfg) {
    case 1: return launch_syrk<64, 64, 2, 2, 4>(P, ldp, C, ldc, nrows, c0, c1, kdim, s);
    case 2: return launch_syrk<128, 64, 2, 2, 3>(P, ldp, C, ldc, nrows, c0, c1, kdim, s);
    default: return launch_syrk<128, 128, 2, 4, 4>(P, ldp, C, ldc, nrows, c0, c1, kdim, s);
    }
}

template <bool AKM, bool BKM>
static void launch_gemm(int64_t m, int64_t n, int64_t k, double alpha, const double *A, int64_t lda,
                        const double *B, int64_t ldb, double beta, double *C, int64_t ldc, char tri, lnb_stream_t s)
{
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(gm::k_gemm_dmma<AKM, BKM>, cudaFuncAttributeMaxDynamicSharedMemorySize, gm::SMEM);
        attr = true;
    }
    dim3 grid((unsigned)((n + gm::BN - 1) / gm::BN), (unsigned)((m + gm::BM - 1) / gm::BM));
    gm::k_gemm_dmma<AKM, BKM><<<grid, gm::THREADS, gm::SMEM, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                  tri);
}

extern "C" int lnb_k_gemm_tri_f64(char ta, char tb, int64_t m, int64_t n, int64_t k, double alpha,
                                  const double *A, int64_t lda, const double *B, int64_t ldb,
                                  double beta, double *C, int64_t ldc, char tri, lnb_stream_t s)
{
    if (m <= 0 || n <= 0) return 0;
    const bool akm = ta == 'N', bkm = tb == 'T';
    if (akm && bkm) launch_gemm<true, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri, s);
    else if (akm) launch_gemm<true, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri, s);
    else if (bkm) launch_gemm<false, true>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri, s);
    else launch_gemm<false, false>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri, s);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

