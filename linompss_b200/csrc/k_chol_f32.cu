// k_chol_f32.cu -- FP32-storage factorization kernels for the low-precision
// factor of the mixed-precision solver (the FP32 twins of the tile tasks:
// task_spotrf / task_strsm / task_ssyrk / task_sgemm, tasks_potrf.c,
// tasks_trsm.c, tasks_syrk.c, task_gemm.c built with -DSINGLE_PRECISION).
//
//   potrf   : leaf diagonal tile in shared memory (k_potrf.cuh)
//   trsm    : panel solve B <- B L^-T, SIMT, rows resident in shared memory,
//             left-looking over 32-column blocks with the leaf's 32x32 inverses;
//             optionally writes the TF32 operand copies of the result for the
//             tensor-core update (hi/lo split x = hi + lo, hi = rna_tf32(x))
//   syrk    : SIMT lower-triangle update (nested diagonal tiles; plain FP32 mode)
//   prep    : column-major panel -> K-major BF16 operand copy scaled by a power
//             of two per 128-row block
//   convert : FP64 A -> FP32 lower triangle with optional symmetric diagonal
//             equilibration  As = S A S,  S = diag(1/sqrt(a_ii))
#include "common.cuh"
#include "k_potrf.cuh"

#include <cuda_bf16.h>

namespace lnb {

LNB_DEV float tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// ------------------------------------------------------------------------
// panel solve X = B L^-T, FP32 SIMT.  A CTA owns 32 rows of the panel and
// walks its 32-column blocks left-looking:
//     acc = B_j - sum_{kc<j} X_kc L_{j,kc}^T ;   X_j = acc Dinv_j^T
// with Dinv_j the leaf's inverse of the j-th 32 x 32 diagonal block.  Each
// (j, kc) chunk stages the L block and the CTA's finished X block (written
// back to B, read again from L2) by cp.async, double-buffered; block starts
// also stage B_j and Dinv_j.  Keeping only the chunk in shared memory (not
// all of X) lets several CTAs share an SM.  64 threads, 4 rows x 4 columns of
// each block per thread, operands by 16-byte shared loads.
// ------------------------------------------------------------------------
namespace ptrsm {
constexpr int LDB = 36;   // padded row of the staged L / Dinv / T blocks
constexpr int NT = 64;    // threads per CTA
}

// dst[k][c] = L[32 j + c][32 kc + k]
LNB_DEV void ptrsm_stage_L(float *dst, const float *L, int64_t lda, int bs, int j, int kc, bool vec, int tid)
{
    for (int idx = tid; idx < 32 * 8; idx += ptrsm::NT) {
        const int k = idx >> 3, c4 = (idx & 7) * 4;
        float *d = dst + k * ptrsm::LDB + c4;
        const int row = 32 * j + c4;
        const float *g = L + row + (int64_t)(32 * kc + k) * lda;
        if (vec && row + 4 <= bs) {
            cp_async16(d, g, true);
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if (row + e < bs) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(d + e)),
                                               "l"(g + e));
                else d[e] = 0.f;
            }
        }
    }
}
// dst[q][c] = Dinv_j[c][q] = dinv[j][c + 32 q]
LNB_DEV void ptrsm_stage_D(float *dst, const float *dinv, int j, int tid)
{
    for (int idx = tid; idx < 32 * 8; idx += ptrsm::NT) {
        const int q = idx >> 3, c4 = (idx & 7) * 4;
        cp_async16(dst + q * ptrsm::LDB + c4, dinv + (int64_t)j * 1024 + c4 + 32 * q, true);
    }
}
// dst[k][r] = B[r0 + r][32 kb + k] (rows past m and columns past bs read as 0).
// From L2 (.cg) when 16-byte aligned; otherwise synchronous L2 loads.
LNB_DEV void ptrsm_stage_B(float *dst, const float *B, int64_t ldb, int64_t m, int bs, int64_t r0, int kb,
                           bool vecB, int tid)
{
    for (int idx = tid; idx < 32 * 8; idx += ptrsm::NT) {
        const int k = idx >> 3, r4 = (idx & 7) * 4;
        float *d = dst + k * 32 + r4;
        const float *g = B + (r0 + r4) + (int64_t)(32 * kb + k) * ldb;
        const int64_t nv64 = (32 * kb + k < bs) ? m - (r0 + r4) : 0;
        const int nv = nv64 < 0 ? 0 : (nv64 > 4 ? 4 : (int)nv64);
        if (vecB) {
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(d)), "l"(nv ? g : B),
                         "r"(4 * nv));
        } else {
#pragma unroll
            for (int e = 0; e < 4; ++e) d[e] = e < nv ? __ldcg(g + e) : 0.f;
        }
    }
}

// 4x4 outer-product accumulate of two 16-byte vectors, acc += sgn x l^T
LNB_DEV void fma4x4(float (&acc)[4][4], const float4 x, const float4 l, float sgn)
{
    const float xv[4] = {sgn * x.x, sgn * x.y, sgn * x.z, sgn * x.w};
    const float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[i][c] = fmaf(xv[i], lv[c], acc[i][c]);
}

__global__ void __launch_bounds__(64) k_trsm_rlt_f32(const float *__restrict__ L, int64_t lda,
                                                     const float *__restrict__ dinv, float *B, int64_t ldb,
                                                     int64_t m, int bs, int vec, float *hi, float *lo, int kpad)
{
    __shared__ __align__(16) float Xc[2][32 * 32];          // staged X_kc, [k][r]
    __shared__ __align__(16) float Lc[2][32 * ptrsm::LDB];  // staged L_{j,kc}, [k][c]
    __shared__ __align__(16) float Ds[2][32 * ptrsm::LDB];  // Dinv_j, [q][c]
    __shared__ __align__(16) float Bs[2][32 * 32];          // B_j, [k][r]
    // finish(j) transposes acc ([q][r]) into the L buffer the finishing chunk
    // has just consumed (34.8 KB per CTA: six CTAs per SM)
    using ptrsm::LDB;
    using ptrsm::NT;
    const int nj = (bs + 31) / 32;
    const int tid = threadIdx.x, rq = tid & 7, cg = tid >> 3;   // rows 4rq..4rq+3, columns 4cg..4cg+3
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const bool vecB = ((uintptr_t)B % 16 == 0) && (ldb % 4 == 0);

    float acc[4][4];
    // X_j = acc Dinv_j^T, written to B and (optionally) as TF32 operands
    auto finish = [&](int j, float *Ts) {
        __syncthreads();                  // every warp is done with the buffer Ts borrows
#pragma unroll
        for (int c = 0; c < 4; ++c)
            *reinterpret_cast<float4 *>(Ts + (4 * cg + c) * LDB + 4 * rq) =
                make_float4(acc[0][c], acc[1][c], acc[2][c], acc[3][c]);
        __syncthreads();
        const float *D = Ds[j & 1];
        float y[4][4] = {};
#pragma unroll 8
        for (int q = 0; q < 32; ++q)
            fma4x4(y, *reinterpret_cast<const float4 *>(Ts + q * LDB + 4 * rq),
                   *reinterpret_cast<const float4 *>(D + q * LDB + 4 * cg), 1.f);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int col = 32 * j + 4 * cg + c;
            if (col < bs)
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    if (r0 + 4 * rq + i < m) B[(r0 + 4 * rq + i) + (int64_t)col * ldb] = y[i][c];
        }
        const int col0 = 32 * j + 4 * cg;
        if (hi != nullptr && col0 < kpad) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t r = r0 + 4 * rq + i;
                if (r < m) {
                    float4 vh, vl;
                    vh.x = tf32_rna(y[i][0]); vh.y = tf32_rna(y[i][1]); vh.z = tf32_rna(y[i][2]); vh.w = tf32_rna(y[i][3]);
                    *reinterpret_cast<float4 *>(hi + r * kpad + col0) = vh;
                    if (lo != nullptr) {
                        vl.x = y[i][0] - vh.x; vl.y = y[i][1] - vh.y; vl.z = y[i][2] - vh.z; vl.w = y[i][3] - vh.w;
                        *reinterpret_cast<float4 *>(lo + r * kpad + col0) = vl;
                    }
                }
            }
        }
    };
    auto load_b = [&](int j) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float4 v = *reinterpret_cast<const float4 *>(Bs[j & 1] + (4 * cg + c) * 32 + 4 * rq);
            acc[0][c] = v.x; acc[1][c] = v.y; acc[2][c] = v.z; acc[3][c] = v.w;
        }
    };
    // chunk (j, kc): the L block and X_kc; a block's first chunk also brings B_j and Dinv_j
    auto stage_chunk = [&](int buf, int j, int kc) {
        ptrsm_stage_L(Lc[buf], L, lda, bs, j, kc, vec, tid);
        ptrsm_stage_B(Xc[buf], B, ldb, m, bs, r0, kc, vecB, tid);
        if (kc == 0) {
            ptrsm_stage_B(Bs[j & 1], B, ldb, m, bs, r0, j, vecB, tid);
            ptrsm_stage_D(Ds[j & 1], dinv, j, tid);
        }
    };

    // block 0: B_0 and Dinv_0, then X_0
    ptrsm_stage_B(Bs[0], B, ldb, m, bs, r0, 0, vecB, tid);
    ptrsm_stage_D(Ds[0], dinv, 0, tid);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    load_b(0);
    finish(0, Lc[0]);                     // nothing is staged in Lc yet
    __syncthreads();                      // X_0 is in B before chunk (1, 0) reads it back
    const int S = nj * (nj - 1) / 2;      // chunks (j, kc), kc < j, in j-major order
    if (S > 0) stage_chunk(0, 1, 0);
    cp_async_commit();
    int j = 1, kc = 0;
    for (int s = 0; s < S; ++s) {
        int jn = j, kn = kc + 1;
        if (kn == jn) { ++jn; kn = 0; }
        // the next chunk's X block is finished: chunk (j', j'-1) is first staged one
        // chunk after block j'-1's finish (for j' >= 2), and (1, 0) above
        if (s + 1 < S) stage_chunk((s + 1) & 1, jn, kn);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        if (kc == 0) load_b(j);
        const float *Lb = Lc[s & 1];
        const float *Xk = Xc[s & 1];
#pragma unroll 8
        for (int k = 0; k < 32; ++k)
            fma4x4(acc, *reinterpret_cast<const float4 *>(Xk + k * 32 + 4 * rq),
                   *reinterpret_cast<const float4 *>(Lb + k * LDB + 4 * cg), -1.f);
        if (kc == j - 1) finish(j, Lc[s & 1]);   // this chunk's L buffer; the next chunk's is the other
        __syncthreads();
        j = jn; kc = kn;
    }
    // operand columns past bs are not written: the update's tensor map ends at
    // K = bs and reads zeros beyond it (kpad may be the stride of a wider array)
    cp_async_wait<0>();
}

// ------------------------------------------------------------------------
// SIMT FP32 lower update C[r,c] -= sum_k P[r,k] P[c,k] (r >= c, c in [c0,c1))
// 64x64 tiles, 256 threads, 4x4 per thread
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_syrk_lower_f32_simt(const float *__restrict__ P, int64_t ldp, float *C,
                                                             int64_t ldc, int64_t nrows, int64_t c0, int64_t c1,
                                                             int kdim)
{
    // K in chunks of 32, staged by cp.async and double-buffered
    __shared__ __align__(16) float As[2][32][68], Bs[2][32][68];
    const int64_t rbase = c0 + (int64_t)blockIdx.y * 64, cbase = c0 + (int64_t)blockIdx.x * 64;
    if (rbase + 64 <= cbase || rbase >= nrows || cbase >= c1) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const bool vec = ((uintptr_t)P % 16 == 0) && (ldp % 4 == 0) && (rbase % 4 == 0) && (cbase % 4 == 0);
    auto stage = [&](int buf, int k0) {
        for (int idx = threadIdx.x; idx < 32 * 16; idx += 256) {
            const int kk = idx >> 4, m4 = (idx & 15) * 4;
            const bool kin = k0 + kk < kdim;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t r = (h ? cbase : rbase) + m4;
                float *d = h ? &Bs[buf][kk][m4] : &As[buf][kk][m4];
                const float *g = P + r + (int64_t)(k0 + kk) * ldp;
                const int64_t nv64 = kin ? nrows - r : 0;
                const int nv = nv64 < 0 ? 0 : (nv64 > 4 ? 4 : (int)nv64);
                if (vec) {
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(d)),
                                 "l"(nv ? g : P), "r"(4 * nv));
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        if (e < nv) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(d + e)),
                                                 "l"(g + e));
                        else d[e] = 0.f;
                    }
                }
            }
        }
    };
    float acc[4][4] = {};
    const int nk = (kdim + 31) / 32;
    stage(0, 0);
    cp_async_commit();
    for (int kt = 0; kt < nk; ++kt) {
        if (kt + 1 < nk) stage((kt + 1) & 1, (kt + 1) * 32);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        const int b = kt & 1;
#pragma unroll 8
        for (int kk = 0; kk < 32; ++kk) {
            float a[4], bb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = As[b][kk][ty + 16 * i]; bb[i] = Bs[b][kk][tx + 16 * i]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
        }
        __syncthreads();
    }
    cp_async_wait<0>();
    float cv[4][4];   // loads first, then stores (avoids serialized read-modify-writes)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t r = rbase + ty + 16 * i, c = cbase + tx + 16 * j;
            cv[i][j] = (r < nrows && c < c1 && r >= c) ? C[r + c * ldc] : 0.f;
        }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t r = rbase + ty + 16 * i, c = cbase + tx + 16 * j;
            if (r < nrows && c < c1 && r >= c) C[r + c * ldc] = cv[i][j] - acc[i][j];
        }
}

// per 128-row block: scale = smallest power of two >= max |x| (1 if the block is zero)
__global__ void __launch_bounds__(256) k_prep_bf16_scale(const float *__restrict__ X, int64_t ldx, int64_t m, int kb,
                                                         float *scale)
{
    __shared__ float red[256];
    const int64_t r0 = (int64_t)blockIdx.x * 128;
    float mx = 0.f;
    for (int idx = threadIdx.x; idx < 128 * kb; idx += 256) {
        const int k = idx / 128, rr = idx % 128;
        const int64_t r = r0 + rr;
        if (r < m) mx = fmaxf(mx, fabsf(X[r + (int64_t)k * ldx]));
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float v = red[0];
        scale[blockIdx.x] = v > 0.f ? exp2f(ceilf(log2f(v))) : 1.f;
    }
}

__global__ void __launch_bounds__(256) k_prep_bf16(const float *__restrict__ X, int64_t ldx, int64_t m, int kb,
                                                   int kpad, const float *__restrict__ scale, __nv_bfloat16 *out)
{
    __shared__ float t[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const int k0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int i = ty; i < 32; i += 8) {
        const int k = k0 + i;
        const int64_t r = r0 + tx;
        t[i][tx] = (k < kb && r < m) ? X[r + (int64_t)k * ldx] : 0.f;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        const int64_t r = r0 + i;
        const int k = k0 + tx;
        if (r < m && k < kpad) out[r * kpad + k] = __float2bfloat16_rn(t[tx][i] / scale[r >> 7]);
    }
}

// ------------------------------------------------------------------------
// conversions
// ------------------------------------------------------------------------
// s[i] = 1/sqrt(a_ii) (or 1 when equilibration is off / a_ii <= 0)
__global__ void k_equil_scale(const double *A, int64_t lda, int64_t n, int on, double *s)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = A[i + i * lda];
        s[i] = (on && d > 0.0) ? 1.0 / sqrt(d) : 1.0;
    }
}

// lower(S A S) in FP32 for columns [c0, c1), rows >= column (column-major,
// ld32), in tiles of 128 rows x 64 columns.  With rsum != NULL the absolute
// values of the FP64 A are summed as well: rsum[i] += |a_ij| for i >= j and
// rsum[j] += |a_ij| for i > j, so that once every column has passed, rsum
// holds the row sums of |A| for the symmetric matrix whose lower triangle A
// stores (its infinity norm is their maximum).  Tile sums are added with FP64
// atomics, so the last bits of rsum depend on their order.
//
// Persistent blocks walk the tiles column tile by column tile (a cursor that
// only moves forward).  Warp w takes columns 8w..8w+7 of a tile and lane l
// rows 2l, 2l+1, 64+2l, 65+2l: all 16 loads of a thread are issued before the
// first use.  vec: A 16-byte aligned with lda even, A32 8-byte aligned with
// ld32 even (pairs of rows move as double2 / float2).
namespace cvt {
constexpr int TR = 128, TC = 64, NT = 256;
}

__global__ void __launch_bounds__(cvt::NT, 3) k_lower_to_f32_t(const double *__restrict__ A, int64_t lda, int64_t n,
                                                           int64_t c0, int64_t c1, const double *__restrict__ s,
                                                           float *__restrict__ A32, int64_t ld32,
                                                           double *__restrict__ rsum, int vec)
{
    __shared__ double red[8][cvt::TR];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r0 = c0 & ~(int64_t)(cvt::TR - 1);
    const int64_t nrt = (n - r0 + cvt::TR - 1) / cvt::TR;
    const int64_t nct = (c1 - c0 + cvt::TC - 1) / cvt::TC;
    int64_t cj = 0, base = 0;
    for (int64_t t = blockIdx.x;; t += gridDim.x) {
        // the column tile holding tile t: column tile cj has the row tiles
        // from the one holding its first column down to the last
        int64_t first;
        for (;;) {
            if (cj >= nct) return;
            first = (c0 + cj * cvt::TC - r0) / cvt::TR;
            if (t < base + nrt - first) break;
            base += nrt - first;
            ++cj;
        }
        const int64_t j0 = c0 + cj * cvt::TC;
        const int64_t i0 = r0 + (first + t - base) * cvt::TR;
        // offsets within the tile: row r = i - i0 is in the triangle and the
        // matrix when lo_c <= r < hi, lo_c = j - i0 for column j (clamped)
        const int hi = n - i0 < cvt::TR ? (int)(n - i0) : cvt::TR;
        const int64_t jw = j0 + warp * 8;
        const int ncol = c1 - jw < 8 ? (int)(c1 - jw) : 8;    // columns of this warp (may be <= 0)
        const int lo0 = jw - i0 < -8 ? -8 : (jw - i0 > cvt::TR ? cvt::TR : (int)(jw - i0));
        const double *pa = A + i0 + jw * lda;
        double si[4], rs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = 64 * (u >> 1) + 2 * lane + (u & 1);
            si[u] = r < hi ? s[i0 + r] : 0.0;
        }
        float *pq = A32 + i0 + jw * ld32;
        // two passes of 4 columns: the loads of a pass are all issued before
        // their first use, and the registers leave room for 3 blocks per SM
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            double v[4][4], sj[4];
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int cc = 4 * p + c4, lo = lo0 + cc;
                sj[c4] = cc < ncol ? s[jw + cc] : 0.0;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = 64 * h + 2 * lane;
                    const bool in0 = cc < ncol && r >= lo && r < hi, in1 = cc < ncol && r + 1 >= lo && r + 1 < hi;
                    const double *q = pa + cc * lda + r;
                    if (vec && in0 && in1) {
                        const double2 w = __ldcs(reinterpret_cast<const double2 *>(q));
                        v[c4][2 * h] = w.x;
                        v[c4][2 * h + 1] = w.y;
                    } else {
                        v[c4][2 * h] = in0 ? __ldcs(q) : 0.0;
                        v[c4][2 * h + 1] = in1 ? __ldcs(q + 1) : 0.0;
                    }
                }
            }
            double cs[4];
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int cc = 4 * p + c4, lo = lo0 + cc;
                cs[c4] = 0.0;
                if (cc >= ncol) continue;                   // warp-uniform
                float o[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = 64 * (u >> 1) + 2 * lane + (u & 1);
                    o[u] = (float)(v[c4][u] * si[u] * sj[c4]);
                    const double a = fabs(v[c4][u]);      // 0 outside the triangle
                    rs[u] += a;
                    if (r > lo) cs[c4] += a;
                }
                float *q = pq + cc * ld32;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = 64 * h + 2 * lane;
                    const bool in0 = r >= lo && r < hi, in1 = r + 1 >= lo && r + 1 < hi;
                    if (vec && in0 && in1) {
                        *reinterpret_cast<float2 *>(q + r) = make_float2(o[2 * h], o[2 * h + 1]);
                    } else {
                        if (in0) q[r] = o[2 * h];
                        if (in1) q[r + 1] = o[2 * h + 1];
                    }
                }
            }
            if (rsum) {
                // the 4 column sums reduced over the warp side by side
#pragma unroll
                for (int d = 16; d > 0; d >>= 1)
#pragma unroll
                    for (int c4 = 0; c4 < 4; ++c4) cs[c4] += __shfl_xor_sync(0xffffffffu, cs[c4], d);
                const double mine = lane == 0 ? cs[0] : lane == 1 ? cs[1] : lane == 2 ? cs[2] : cs[3];
                if (lane < 4 && 4 * p + lane < ncol && mine != 0.0) atomicAdd(rsum + jw + 4 * p + lane, mine);
            }
        }
        if (rsum) {
#pragma unroll
            for (int u = 0; u < 4; ++u) red[warp][64 * (u >> 1) + 2 * lane + (u & 1)] = rs[u];
            __syncthreads();
            if (threadIdx.x < cvt::TR) {
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < 8; ++w) sum += red[w][threadIdx.x];
                if ((int)threadIdx.x < hi && sum != 0.0) atomicAdd(rsum + i0 + threadIdx.x, sum);
            }
            __syncthreads();
        }
    }
}

static int launch_lower_to_f32(const double *A, int64_t lda, int64_t n, int64_t c0, int64_t c1, const double *S,
                               float *A32, int64_t ld32, double *rsum, cudaStream_t s)
{
    static int slots = 0;      // resident blocks on the whole GPU
    if (!slots) {
        int dev = 0, sms = 148, per = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_lower_to_f32_t, cvt::NT, 0);
        slots = sms * (per > 0 ? per : 1);
    }
    const int vec = ((uintptr_t)A % 16 == 0) && (lda % 2 == 0) && ((uintptr_t)A32 % 8 == 0) && (ld32 % 2 == 0);
    const int64_t r0 = c0 & ~(int64_t)(cvt::TR - 1);
    const int64_t tiles = ((n - r0 + cvt::TR - 1) / cvt::TR) * ((c1 - c0 + cvt::TC - 1) / cvt::TC);
    const int64_t grid = tiles < slots ? tiles : slots;
    k_lower_to_f32_t<<<(unsigned)grid, cvt::NT, 0, s>>>(A, lda, n, c0, c1, S, A32, ld32, rsum, vec);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

}  // namespace lnb

using namespace lnb;

extern "C" int lnb_k_lower_to_f32_cols(const double *A, int64_t lda, int64_t n, int64_t c0, int64_t c1,
                                       const double *S, float *A32, int64_t ld32, double *rsum, lnb_stream_t s)
{
    if (c1 <= c0 || c0 >= n) return 0;
    return launch_lower_to_f32(A, lda, n, c0, c1 < n ? c1 : n, S, A32, ld32, rsum, s);
}

extern "C" int lnb_k_equil_scale_vec(const double *a, int64_t n, int on, double *s_out, lnb_stream_t s)
{
    if (n <= 0) return 0;
    k_equil_scale<<<(unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), 256, 0, s>>>(a, 0, n, on, s_out);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_potrf_f32(float *A, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                               lnb_stream_t s)
{
    if (bs <= 0) return 0;
    if (bs > LEAF) return (int)cudaErrorInvalidValue;
    const int smem = (int)leaf_smem_bytes<float>(bs);
    cudaFuncSetAttribute(k_potrf_leaf<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_potrf_leaf<float><<<1, 256, smem, s>>>(A, lda, bs, row0, dinv, st);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_trsm_rlt_f32(const float *L, int64_t lda, const float *dinv, float *B, int64_t ldb, int64_t m,
                                  int bs, lnb_stream_t s)
{
    if (m <= 0 || bs <= 0) return 0;
    const int vec = ((uintptr_t)L % 16 == 0) && (lda % 4 == 0);
    k_trsm_rlt_f32<<<(unsigned)((m + 31) / 32), ptrsm::NT, 0, s>>>(L, lda, dinv, B, ldb, m, bs, vec, nullptr,
                                                                    nullptr, 0);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

// the panel solve plus the K-major TF32 operand copies of its result (hi, and
// lo = x - hi when lo != NULL), row stride kpad >= 32 ceil(bs/32), a multiple
// of 4, hi/lo 16-byte aligned; K columns [0, 32 ceil(bs/32)) of each row are
// written, nothing beyond
extern "C" int lnb_k_trsm_rlt_prep_f32(const float *L, int64_t lda, const float *dinv, float *B, int64_t ldb,
                                       int64_t m, int bs, float *hi, float *lo, int kpad, lnb_stream_t s)
{
    if (m <= 0 || bs <= 0) return 0;
    const int nj = (bs + 31) / 32;
    if (32 * nj > kpad || kpad % 4 || (uintptr_t)hi % 16 || (uintptr_t)lo % 16) return (int)cudaErrorInvalidValue;
    const int vec = ((uintptr_t)L % 16 == 0) && (lda % 4 == 0);
    k_trsm_rlt_f32<<<(unsigned)((m + 31) / 32), ptrsm::NT, 0, s>>>(L, lda, dinv, B, ldb, m, bs, vec, hi, lo, kpad);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_syrk_lower_f32_simt(const float *P, int64_t ldp, float *C, int64_t ldc, int64_t nrows,
                                         int64_t c0, int64_t c1, int kdim, lnb_stream_t s)
{
    if (nrows <= c0 || c1 <= c0 || kdim <= 0) return 0;
    dim3 grid((unsigned)((c1 - c0 + 63) / 64), (unsigned)((nrows - c0 + 63) / 64));
    k_syrk_lower_f32_simt<<<grid, 256, 0, s>>>(P, ldp, C, ldc, nrows, c0, c1, kdim);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_prep_bf16(const float *X, int64_t ldx, int64_t m, int kb, int kpad, float *scale, void *out,
                               lnb_stream_t s)
{
    if (m <= 0) return 0;
    k_prep_bf16_scale<<<(unsigned)((m + 127) / 128), 256, 0, s>>>(X, ldx, m, kb, scale);
    lnb_prof_count(1);
    dim3 grid((unsigned)((m + 31) / 32), (unsigned)((kpad + 31) / 32));
    k_prep_bf16<<<grid, 256, 0, s>>>(X, ldx, m, kb, kpad, scale, (__nv_bfloat16 *)out);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_lower_to_f32(const double *A, int64_t lda, int64_t n, int equilibrate, double *s_out,
                                  float *A32, int64_t ld32, double *rsum, lnb_stream_t s)
{
    if (n <= 0) return 0;
    k_equil_scale<<<(unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), 256, 0, s>>>(A, lda, n, equilibrate,
                                                                                             s_out);
    lnb_prof_count(1);
    return launch_lower_to_f32(A, lda, n, 0, n, s_out, A32, ld32, rsum, s);
}

// ------------------------------------------------------------------------
// FP64 refactor of a failed low-precision diagonal tile
// ------------------------------------------------------------------------
namespace lnb {
// T[r,c] = s_r A[r,c] s_c for r >= c (bs x bs, FP64, ld ldt)
__global__ void k_scaled_tile_f64(const double *A, int64_t lda, const double *s, int bs, double *T, int64_t ldt)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < bs * bs; idx += gridDim.x * blockDim.x) {
        const int c = idx / bs, r = idx % bs;
        if (r >= c) T[r + (int64_t)c * ldt] = s[r] * A[r + (int64_t)c * lda] * s[c];
    }
}
// D (m x k, FP64, ld ldd) = X (FP32, ld ldx)
__global__ void k_f32_to_f64(const float *X, int64_t ldx, int64_t m, int64_t k, double *D, int64_t ldd)
{
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < m * k;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = idx / m, r = idx % m;
        D[r + c * ldd] = (double)X[r + c * ldx];
    }
}
// lower triangle of the FP64 tile back into FP32
__global__ void k_f64_to_f32_lower(const double *T, int64_t ldt, int bs, float *X, int64_t ldx)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < bs * bs; idx += gridDim.x * blockDim.x) {
        const int c = idx / bs, r = idx % bs;
        if (r >= c) X[r + (int64_t)c * ldx] = (float)T[r + (int64_t)c * ldt];
    }
}
// T[i,i] += shift; also copies src -> T first when src != NULL (lower part)
__global__ void k_restore_shift(const double *src, double *T, int64_t ldt, int bs, double shift)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < bs * bs; idx += gridDim.x * blockDim.x) {
        const int c = idx / bs, r = idx % bs;
        if (r >= c) T[r + (int64_t)c * ldt] = src[r + (int64_t)c * ldt] + (r == c ? shift : 0.0);
    }
}
// max |T[i,i]| into out[0] (one CTA)
__global__ void k_diag_absmax(const double *T, int64_t ldt, int bs, double *out)
{
    __shared__ double red[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < bs; i += 256) m = fmax(m, fabs(T[i + (int64_t)i * ldt]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}
// inverses of the 32x32 diagonal blocks of an FP32 factored tile (warp per block)
__global__ void k_dinv32_f32(const float *L, int64_t ldl, int bs, float *dinv)
{
    __shared__ float X[32][33];
    const int q = blockIdx.x, c = threadIdx.x, o = q * 32;
    const int qn = bs - o < 32 ? bs - o : 32;
    for (int r = 0; r < 32; ++r) {
        float v;
        if (c >= qn) v = (r == c) ? 1.f : 0.f;
        else if (r < c || r >= qn) v = 0.f;
        else if (r == c) v = 1.f / L[(o + c) + (int64_t)(o + c) * ldl];
        else {
            float s = 0.f;
            for (int p = c; p < r; ++p) s += L[(o + r) + (int64_t)(o + p) * ldl] * X[p][c];
            v = -s / L[(o + r) + (int64_t)(o + r) * ldl];
        }
        X[r][c] = v;
        __syncwarp();
    }
    for (int r = 0; r < 32; ++r) dinv[(int64_t)q * 1024 + r + 32 * c] = X[r][c];
}
}  // namespace lnb

static unsigned g1(int64_t work) { int64_t b = (work + 255) / 256; return (unsigned)(b < 4096 ? (b > 0 ? b : 1) : 4096); }

extern "C" int lnb_k_scaled_tile_f64(const double *A, int64_t lda, const double *s, int bs, double *T, int64_t ldt,
                                     lnb_stream_t st)
{
    k_scaled_tile_f64<<<g1((int64_t)bs * bs), 256, 0, st>>>(A, lda, s, bs, T, ldt);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
extern "C" int lnb_k_f32_to_f64(const float *X, int64_t ldx, int64_t m, int64_t k, double *D, int64_t ldd,
                                lnb_stream_t st)
{
    if (m <= 0 || k <= 0) return 0;
    k_f32_to_f64<<<g1(m * k), 256, 0, st>>>(X, ldx, m, k, D, ldd);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
extern "C" int lnb_k_f64_to_f32_lower(const double *T, int64_t ldt, int bs, float *X, int64_t ldx, lnb_stream_t st)
{
    k_f64_to_f32_lower<<<g1((int64_t)bs * bs), 256, 0, st>>>(T, ldt, bs, X, ldx);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
extern "C" int lnb_k_restore_shift(const double *src, double *T, int64_t ldt, int bs, double shift, lnb_stream_t st)
{
    k_restore_shift<<<g1((int64_t)bs * bs), 256, 0, st>>>(src, T, ldt, bs, shift);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
extern "C" int lnb_k_diag_absmax(const double *T, int64_t ldt, int bs, double *out, lnb_stream_t st)
{
    k_diag_absmax<<<1, 256, 0, st>>>(T, ldt, bs, out);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
extern "C" int lnb_k_dinv32_f32(const float *L, int64_t ldl, int bs, float *dinv, lnb_stream_t st)
{
    k_dinv32_f32<<<(unsigned)((bs + 31) / 32), 32, 0, st>>>(L, ldl, bs, dinv);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

namespace lnb {
__global__ void k_f64_to_f32(const double *D, int64_t ldd, int64_t m, int64_t k, float *X, int64_t ldx)
{
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < m * k;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = idx / m, r = idx % m;
        X[r + c * ldx] = (float)D[r + c * ldd];
    }
}
}  // namespace lnb

extern "C" int lnb_k_f64_to_f32(const double *D, int64_t ldd, int64_t m, int64_t k, float *X, int64_t ldx,
                                lnb_stream_t st)
{
    if (m <= 0 || k <= 0) return 0;
    k_f64_to_f32<<<g1(m * k), 256, 0, st>>>(D, ldd, m, k, X, ldx);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
