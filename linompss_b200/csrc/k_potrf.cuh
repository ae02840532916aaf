// k_potrf.cuh -- diagonal-tile Cholesky leaf kernel (FP64 and FP32).
//
// Semantics of task_dpotrf / LAPACK potrf 'L' (tasks_potrf.c:20-24) on a
// tile of order bs <= 128, with the info the reference drops reported in
// the status word.  Larger diagonal tiles are factored by the host-side
// nested schedule (leaf POTRF + panel TRSM + update on 128-wide sub-tiles),
// the structure of the reference's nested variant (chol_nrlmain.c).
//
// The whole tile lives in shared memory and is factored in 32-column panels:
//   (1) all threads factor the 32 x 32 diagonal block right-looking and build
//       its inverse in the same sweep, one barrier per column (one-warp
//       versions of both were the leaf's serial bottleneck); columns are
//       scaled by rsqrt(pivot), the reciprocal LAPACK's potf2 scales by.
//   (2) the rows below the block become b * inv(L_jj)^T: independent dot
//       products, 4 threads per row, instead of a substitution chain;
//   (3) the rank-32 update of the trailing triangle reads a transposed copy
//       of the panel with vector loads, 4 x 4 outputs per thread.
// The 32 x 32 inverses are written out (dinv) for the panel TRSM below the
// tile.  After a failed pivot the columns before it are finished for every
// row of the tile, the failing diagonal keeps its updated value, and the
// inverses use the identity past the failure.
#pragma once
#include "common.cuh"

namespace lnb {

constexpr int LEAF = 128;   // max order of a leaf tile
constexpr int LP = 32;      // panel width of the leaf factorization

LNB_DEV void leaf_cp_async(float *smem, const float *g)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem)), "l"(g));
}
LNB_DEV void leaf_cp_async(double *smem, const double *g) { cp_async8(smem, g, true); }
LNB_DEV float leaf_rsqrt(float x) { return rsqrtf(x); }
LNB_DEV double leaf_rsqrt(double x) { return rsqrt(x); }

// shared memory layout of the leaf (offsets in elements of T, 16-byte aligned)
struct LeafLayout {
    int lds, ldp;
    size_t s_off, p_off, li_off, rd_off, total;
};
template <typename T>
__host__ __device__ inline LeafLayout leaf_layout(int bs)
{
    LeafLayout L;
    const int v = 16 / (int)sizeof(T);
    L.lds = bs + 1;
    L.ldp = ((bs + 3) / 4) * 4 + 4;   // 4-row vector reads may run 3 past bs
    L.s_off = 0;
    L.p_off = (((size_t)bs * L.lds + v - 1) / v) * v;
    L.li_off = L.p_off + (size_t)LP * L.ldp;
    L.rd_off = L.li_off + ((LP * (LP + 1) + v - 1) / v) * v;
    L.total = L.rd_off + 2 * LP;
    return L;
}

template <typename T>
__global__ void __launch_bounds__(256) k_potrf_leaf(T *A, int64_t lda, int bs, int64_t row0, T *dinv,
                                                    lnb_status_t *st)
{
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const LeafLayout LY = leaf_layout<T>(bs);
    const int LDS = LY.lds, LDP = LY.ldp;
    T *base = reinterpret_cast<T *>(sm_raw);
    T *S = base + LY.s_off;     // S[r * LDS + c] = A[r, c], lower part
    T *Pt = base + LY.p_off;    // Pt[p * LDP + r] = L[r, j0 + p]: the panel below the block, transposed
    T *Li = base + LY.li_off;   // Li[p * 33 + j] = inv(L_jj)[j][p]
    T *Rd = base + LY.rd_off;   // Rd[c] = rsqrt(pivot c) = 1 / L[c][c]; Rd[LP + c] = pivot c
    __shared__ int fail_col;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) fail_col = bs;

    // the tile arrives by element-wise cp.async, all copies in flight at once
    // (a plain load loop would pay one memory round trip per iteration)
    for (int idx = tid; idx < bs * bs; idx += blockDim.x) {
        const int c = idx / bs, r = idx - c * bs;
        if (r >= c) leaf_cp_async(S + r * LDS + c, A + (int64_t)r + (int64_t)c * lda);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    for (int j0 = 0; j0 < bs; j0 += LP) {
        const int jb = min(LP, bs - j0);
        // ---- (1) factor the jb x jb diagonal block right-looking with all threads,
        //      one barrier per column, and build its inverse X = inv(L_jj) in the
        //      same sweep (X = I; for each column c: X[r][:] -= L[r][c] X[c][:] / L[c][c]
        //      for r > c).  Both use the unscaled column over the pivot, e.g.
        //      S[r][cc] -= S[r][c] S[cc][c] / d_c; the scaling of L's column c and of
        //      X's row c by rsqrt(d_c) (the reciprocal potf2 uses) waits for one pass
        //      at the end.  X lives in Li (Li[q][r] = X[r][q]). ----
        {
            const int ty = tid >> 5, tx = lane;
            for (int idx = tid; idx < LP * (LP + 1); idx += blockDim.x) {
                const int q = idx / (LP + 1), r = idx - q * (LP + 1);
                Li[idx] = (r == q) ? T(1) : T(0);
            }
            __syncthreads();
            int fc = jb;
            for (int c = 0; c < jb; ++c) {
                const T d = S[(j0 + c) * LDS + j0 + c];       // every thread reads the same pivot
                if (!(d > T(0))) { fc = c; break; }            // potf2 keeps the updated pivot
                const T inv = leaf_rsqrt(d);
                const T invd = inv * inv;
                if (tid == 0) { Rd[c] = inv; Rd[LP + c] = d; }
                // thread (ty, tx): rows r = c+1+ty+8u (u < 4) of column cc = c+1+tx of L,
                // and of column q = tx of X; all loads issued before the updates
                const int cc = c + 1 + tx;
                T lr[4], sv[4], xv[4];
                const T lcc = cc < jb ? S[(j0 + cc) * LDS + j0 + c] * invd : T(0);
                const T xcq = tx <= c ? Li[tx * (LP + 1) + c] * invd : T(0);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = c + 1 + ty + 8 * u;
                    const bool in = r < jb;
                    lr[u] = in ? S[(j0 + r) * LDS + j0 + c] : T(0);
                    sv[u] = (in && cc < jb && r >= cc) ? S[(j0 + r) * LDS + j0 + cc] : T(0);
                    xv[u] = (in && tx <= c) ? Li[tx * (LP + 1) + r] : T(0);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = c + 1 + ty + 8 * u;
                    if (r < jb && cc < jb && r >= cc) S[(j0 + r) * LDS + j0 + cc] = sv[u] - lr[u] * lcc;
                    // X rows r > c, column q = tx <= c: X[r][q] -= S[r][c] X[c][q] / d_c
                    if (r < jb && tx <= c) Li[tx * (LP + 1) + r] = xv[u] - lr[u] * xcq;
                }
                __syncthreads();
            }
            if (tid == 0 && fc < jb) {
                fail_col = j0 + fc;
                atomicCAS(&st->info, 0, (int)(row0 + j0 + fc + 1));
            }
            // scale L's columns and X's rows (X = identity past a failed pivot)
            for (int idx = tid; idx < jb * jb; idx += blockDim.x) {
                const int r = idx / jb, c = idx - r * jb;
                if (c < fc && r >= c) {
                    T &v = S[(j0 + r) * LDS + j0 + c];
                    v = (r == c) ? Rd[LP + c] * Rd[c] : v * Rd[c];
                }
            }
            for (int idx = tid; idx < LP * LP; idx += blockDim.x) {
                const int r = idx / LP, q = idx - r * LP;      // X[r][q]
                T &x = Li[q * (LP + 1) + r];
                if (r < fc) x *= Rd[r];
                else x = (r == q) ? T(1) : T(0);
            }
            __syncthreads();
            if (dinv != nullptr) {
                T *D = dinv + (int64_t)(j0 / LP) * LP * LP;
                for (int idx = tid; idx < LP * LP; idx += blockDim.x) {
                    const int c = idx / LP, r = idx - c * LP;
                    D[r + LP * c] = Li[c * (LP + 1) + r];
                }
            }
        }
        __syncthreads();
        // columns of this panel that are final for the rows below
        const int jv = fail_col < bs ? fail_col - j0 : jb;
        // ---- (2) rows below the block: x_r = b_r inv(L_jj)^T, 4 threads per row ----
        const int t0 = j0 + jb;
        const int g = tid & 3;
        for (int rb = t0; rb < bs; rb += 64) {
            const int r = rb + (tid >> 2);
            const bool act = r < bs;
            T b[LP];
#pragma unroll
            for (int p = 0; p < LP; ++p) b[p] = (act && p < jb) ? S[r * LDS + j0 + p] : T(0);
            __syncwarp();
            T acc[LP / 4];
#pragma unroll
            for (int s = 0; s < LP / 4; ++s) acc[s] = T(0);
#pragma unroll
            for (int p = 0; p < LP; ++p)
#pragma unroll
                for (int s = 0; s < LP / 4; ++s) acc[s] = fma(b[p], Li[p * (LP + 1) + g + 4 * s], acc[s]);
#pragma unroll
            for (int s = 0; s < LP / 4; ++s) {
                const int j = g + 4 * s;
                if (act && j < jv) {
                    S[r * LDS + j0 + j] = acc[s];
                    Pt[j * LDP + r] = acc[s];
                }
            }
        }
        __syncthreads();
        if (fail_col < bs) break;
        // ---- (3) rank-jb update of the trailing lower triangle, 4x4 per thread ----
        const int tr = bs - t0;
        if (tr > 0) {
            const int nb4 = (tr + 3) / 4, nblk = nb4 * (nb4 + 1) / 2;
            for (int id = tid; id < nblk; id += blockDim.x) {
                int bi = (int)((sqrtf(8.0f * id + 1.0f) - 1.0f) * 0.5f);
                while (bi * (bi + 1) / 2 > id) --bi;
                while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
                const int bj = id - bi * (bi + 1) / 2;
                const int ra = t0 + 4 * bi, rc = t0 + 4 * bj;
                T acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
                for (int p = 0; p < jb; ++p) {
                    T a[4], c[4];
                    if constexpr (sizeof(T) == 4) {
                        const float4 va = *reinterpret_cast<const float4 *>(Pt + p * LDP + ra);
                        const float4 vc = *reinterpret_cast<const float4 *>(Pt + p * LDP + rc);
                        a[0] = va.x; a[1] = va.y; a[2] = va.z; a[3] = va.w;
                        c[0] = vc.x; c[1] = vc.y; c[2] = vc.z; c[3] = vc.w;
                    } else {
                        const double2 va0 = *reinterpret_cast<const double2 *>(Pt + p * LDP + ra);
                        const double2 va1 = *reinterpret_cast<const double2 *>(Pt + p * LDP + ra + 2);
                        const double2 vc0 = *reinterpret_cast<const double2 *>(Pt + p * LDP + rc);
                        const double2 vc1 = *reinterpret_cast<const double2 *>(Pt + p * LDP + rc + 2);
                        a[0] = va0.x; a[1] = va0.y; a[2] = va1.x; a[3] = va1.y;
                        c[0] = vc0.x; c[1] = vc0.y; c[2] = vc1.x; c[3] = vc1.y;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], c[j], acc[i][j]);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int r = ra + i, cc = rc + j;
                        if (r < bs && cc < bs && r >= cc) S[r * LDS + cc] -= acc[i][j];
                    }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    // write the lower triangle back (past a failed pivot, the partial state)
    for (int idx = tid; idx < bs * bs; idx += blockDim.x) {
        const int c = idx / bs, r = idx - c * bs;
        if (r >= c) A[(int64_t)r + (int64_t)c * lda] = S[r * LDS + c];
    }
    // blocks of the tile after a failed panel: identity inverses
    if (dinv != nullptr) {
        const int nq = (bs + LP - 1) / LP;
        const int q0 = fail_col < bs ? fail_col / LP + 1 : nq;
        for (int idx = tid; idx < (nq - q0) * LP * LP; idx += blockDim.x) {
            const int q = q0 + idx / (LP * LP), e = idx % (LP * LP);
            dinv[(int64_t)q * LP * LP + e] = (e % LP == e / LP) ? T(1) : T(0);
        }
    }
}

template <typename T>
inline size_t leaf_smem_bytes(int bs)
{
    return leaf_layout<T>(bs).total * sizeof(T);
}

}  // namespace lnb
