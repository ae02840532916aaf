// k_potrf.cuh -- diagonal-tile Cholesky leaf kernel (FP64 and FP32).
//
// Semantics of task_dpotrf / LAPACK potrf 'L' (tasks_potrf.c:20-24) on a
// tile of order bs <= 128, with the info the reference drops reported in
// the status word.  Larger diagonal tiles are factored by the host-side
// nested schedule (leaf POTRF + panel TRSM + DMMA update on 128-wide
// sub-tiles), the structure of the reference's nested variant
// (chol_nrlmain.c).
//
// The whole tile lives in shared memory (128 x 129 doubles = 129 KB).  For
// each 16-column panel, warp 0 factors the 16 x 16 diagonal block in
// registers with shuffles; then all threads solve the rows below it (one row
// per thread) and apply the rank-16 update to the trailing lower triangle.  At the
// end the inverses of the tile's 32x32 diagonal blocks (used by the panel
// TRSM) are computed from the factor in shared memory.
#pragma once
#include "common.cuh"

namespace lnb {

constexpr int LEAF = 128;   // max order of a leaf tile
constexpr int LP = 16;      // panel width of the leaf factorization

template <typename T>
__global__ void __launch_bounds__(256) k_potrf_leaf(T *A, int64_t lda, int bs, int64_t row0, T *dinv,
                                                    lnb_status_t *st)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int LDS = bs + 1;
    T *S = reinterpret_cast<T *>(sm_raw);  // S[r * LDS + c] = A[r, c], lower part
    __shared__ int fail_col;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) fail_col = bs;

    for (int idx = tid; idx < bs * bs; idx += blockDim.x) {
        const int c = idx / bs, r = idx - c * bs;
        if (r >= c) S[r * LDS + c] = A[(int64_t)r + (int64_t)c * lda];
    }
    __syncthreads();

    for (int j0 = 0; j0 < bs; j0 += LP) {
        const int jb = min(LP, bs - j0);
        if (warp == 0) {
            // (1) the jb x jb diagonal block in registers: lane l holds row j0+l
            T x[LP];
#pragma unroll
            for (int c = 0; c < LP; ++c)
                x[c] = (lane < jb && c < jb && lane >= c) ? S[(j0 + lane) * LDS + j0 + c] : T(0);
            int bad = bs;
#pragma unroll
            for (int c = 0; c < LP; ++c) {
                if (c < jb && bad == bs) {
                    const T d = __shfl_sync(0xffffffffu, x[c], c);
                    if (!(d > T(0))) {
                        bad = j0 + c;
                    } else {
                        const T dd = sqrt(d);
                        if (lane == c) x[c] = dd;
                        else if (lane > c) x[c] = x[c] / dd;
#pragma unroll
                        for (int cc = c + 1; cc < LP; ++cc) {
                            const T l = __shfl_sync(0xffffffffu, x[c], cc);   // L[j0+cc][j0+c]
                            if (lane >= cc) x[cc] -= x[c] * l;
                        }
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < LP; ++c)
                if (lane < jb && c < jb && lane >= c) S[(j0 + lane) * LDS + j0 + c] = x[c];
            if (lane == 0 && bad < bs) {
                fail_col = bad;
                atomicCAS(&st->info, 0, (int)(row0 + bad + 1));
            }
        }
        __syncthreads();
        // after a failed pivot only the columns before it are finished, for
        // every row of the tile (as LAPACK's column-by-column potf2 leaves them)
        const int jv = fail_col < bs ? fail_col - j0 : jb;
        // (2) rows below the diagonal block: X = B L^-T, one row per thread,
        //     L read from shared memory (the same element by all threads)
        for (int r = j0 + jb + tid; r < bs; r += blockDim.x) {
            T x[LP];
#pragma unroll
            for (int c = 0; c < LP; ++c) {
                if (c < jv) {
                    T v = S[r * LDS + j0 + c];
#pragma unroll
                    for (int p = 0; p < c; ++p) v -= x[p] * S[(j0 + c) * LDS + j0 + p];
                    x[c] = v / S[(j0 + c) * LDS + j0 + c];
                    S[r * LDS + j0 + c] = x[c];
                }
            }
        }
        __syncthreads();
        if (fail_col < bs) break;
        // rank-jb update of the trailing lower triangle, 4x4 blocks per thread
        const int t0 = j0 + jb, tr = bs - t0;
        if (tr > 0) {
            const int nb4 = (tr + 3) / 4, nblk = nb4 * (nb4 + 1) / 2;
            for (int id = tid; id < nblk; id += blockDim.x) {
                int bi = (int)((sqrtf(8.0f * id + 1.0f) - 1.0f) * 0.5f);
                while (bi * (bi + 1) / 2 > id) --bi;
                while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
                const int bj = id - bi * (bi + 1) / 2;
                const int ra = t0 + 4 * bi, rb = t0 + 4 * bj;
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
                for (int p = 0; p < jb; ++p) {
                    T a[4], b[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        a[i] = (ra + i < bs) ? S[(ra + i) * LDS + j0 + p] : T(0);
                        b[i] = (rb + i < bs) ? S[(rb + i) * LDS + j0 + p] : T(0);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int r = ra + i, c = rb + j;
                        if (r < bs && c < bs && r >= c) S[r * LDS + c] -= acc[i][j];
                    }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    const int lim = fail_col;
    // write the factored lower triangle back (columns < lim are the factor;
    // past a failed pivot the partial state is written like LAPACK does)
    for (int idx = tid; idx < bs * bs; idx += blockDim.x) {
        const int c = idx / bs, r = idx - c * bs;
        if (r >= c) A[(int64_t)r + (int64_t)c * lda] = S[r * LDS + c];
    }
    // inverses of the 32x32 diagonal blocks (identity past a failed pivot):
    // warp q inverts block q, lane c builds column c in shared scratch
    if (dinv != nullptr) {
        T *X = S + bs * LDS;                        // 4 x [32][33] scratch after the tile
        const int nq = (bs + 31) / 32;
        for (int q = warp; q < nq; q += blockDim.x / 32) {
            const int qn = max(0, min(32, lim - q * 32));
            T *Xq = X + (q & 3) * 32 * 33;
            const int c = lane, o = q * 32;
            for (int r = 0; r < 32; ++r) {
                T v;
                if (c >= qn) v = (r == c) ? T(1) : T(0);
                else if (r < c || r >= qn) v = T(0);
                else if (r == c) v = T(1) / S[(o + c) * LDS + o + c];
                else {
                    T s = T(0);
                    for (int p = c; p < r; ++p) s += S[(o + r) * LDS + o + p] * Xq[p * 33 + c];
                    v = -s / S[(o + r) * LDS + o + r];
                }
                Xq[r * 33 + c] = v;
            }
            __syncwarp();
            T *D = dinv + (int64_t)q * 1024;
            for (int r = 0; r < 32; ++r) D[r + 32 * c] = Xq[r * 33 + c];
            __syncwarp();
        }
    }
}

}  // namespace lnb
