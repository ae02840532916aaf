// k_potrf_cluster.cu -- FP32 Cholesky of one diagonal tile of order bs <= 512
// (bs % 32 == 0) by a cluster of 8 CTAs, the tile resident in their shared
// memory for the whole factorization.
//
// A diagonal tile factored by one CTA is a chain of 32-column steps on one SM;
// split over separate launches, every launch waits for an SM that the trailing
// update of the outer factorization holds.  Here the 32 x 32 blocks of the
// tile's lower triangle are distributed over the cluster by block rows (CTA q
// owns block rows q and 15 - q, so every CTA holds 17 blocks), and each
// 32-column step j runs as
//   (a) the owner of block row j factors its diagonal block in registers and
//       forms X = L_jj^-1, which it stores into every CTA's shared memory;
//   (c) every CTA solves its blocks below: L_ij = A_ij X^T, kept in its own
//       slot and stored into every CTA's panel buffer (distributed shared
//       memory);
//   (e) every CTA updates its blocks A_ik -= L_ij L_kj^T, k in (j, i]; the
//       owner of block row j + 1 updates that diagonal block first and factors
//       it (step (a) of j + 1) while its other warps continue the update.
// Hardware cluster barriers separate the phases; there is no spin-wait.  The
// sweep stores nothing to global memory (each barrier's release would wait for
// such stores); the finished blocks and the per-block inverses X (dinv,
// column-major 32 x 32 each, for the panel solve that follows) are written out
// after it.
//
// Algorithm: right-looking blocked Cholesky as in the reference's tile
// schedule (src/chol_rl.c, POTRF/TRSM/SYRK/GEMM per step), applied inside one
// tile of the outer factorization.
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace lnb {

constexpr int PCS = 8;               // CTAs per cluster
constexpr int PNB = 2 * PCS;         // 32-wide blocks per tile side, at most
constexpr int PNT = 256;             // threads per CTA
constexpr int PBK = 32 * 32;         // floats in one block
constexpr int PXS = 36;              // column stride of the shared inverse (conflict-free stores)
constexpr int POWN = 2 * PCS + 1;    // blocks owned per CTA (rows q and 2 PCS - 1 - q)
constexpr int PC_SMEM = ((POWN + PNB) * PBK + 3 * 32 * PXS + 32) * 4 + 16;

LNB_DEV int pc_owner(int i) { return i < PCS ? i : 2 * PCS - 1 - i; }
// shared-memory slot of block (i, k), k <= i, in its owner q
LNB_DEV int pc_slot(int i, int k, int q) { return i < PCS ? k : q + 1 + k; }

// Right-looking Cholesky of the 32 x 32 block D (column-major) by one warp,
// lane r holding row r in registers.  D receives L (entries above the diagonal
// keep unused values), rv[c] = 1 / L[c][c].  Returns 0 or the 1-based column of
// the first non-positive pivot.
LNB_DEV int pc_factor_block(float *D, float *rv, int lane)
{
    // dd[cc]: every lane's copy of the diagonal entry lane cc holds in a[cc].
    // It takes the same fma(-x, x, .) with the broadcast x = L[cc][c] as lane
    // cc's own entry, so it is bit-identical, and the next pivot needs no
    // shuffle on the chain of 32 dependent columns.
    float a[32], dd[32];
#pragma unroll
    for (int c = 0; c < 32; ++c) {
        a[c] = D[c * 32 + lane];
        dd[c] = D[c * 32 + c];
    }
    int bad = 0;
#pragma unroll
    for (int c = 0; c < 32; ++c) {
        const float d = dd[c];
        if (bad == 0 && !(d > 0.f)) bad = c + 1;
        const float s = rsqrtf(d);
        a[c] = (lane == c) ? d * s : a[c] * s;
        if (lane == 0) rv[c] = s;
#pragma unroll
        for (int cc = c + 1; cc < 32; ++cc) {
            const float x = __shfl_sync(0xffffffffu, a[c], cc);
            a[cc] = fmaf(-a[c], x, a[cc]);
            dd[cc] = fmaf(-x, x, dd[cc]);
        }
    }
#pragma unroll
    for (int c = 0; c < 32; ++c) D[c * 32 + lane] = a[c];
    __syncwarp();
    return bad;
}

// X = L^-1 by forward substitution, lane q building column q: x[p] = X[p][q]
LNB_DEV void pc_inverse(const float *D, const float *rv, int lane, float (&x)[32])
{
#pragma unroll
    for (int p = 0; p < 32; ++p) {
        float s0 = (p == lane) ? 1.f : 0.f, s1 = 0.f;
#pragma unroll
        for (int m = 0; m + 1 < p; m += 2) {
            s0 = fmaf(-D[m * 32 + p], x[m], s0);
            s1 = fmaf(-D[(m + 1) * 32 + p], x[m + 1], s1);
        }
        if (p & 1) s0 = fmaf(-D[(p - 1) * 32 + p], x[p - 1], s0);
        x[p] = (s0 + s1) * rv[p];
    }
}

// C -= P1 P2^T for 32 x 32 column-major blocks, one warp; lane tile 4 rows x 8 columns
LNB_DEV void pc_update(float *C, const float *P1, const float *P2, int lane)
{
    const int r0 = 4 * (lane & 7), c0 = 8 * (lane >> 3);
    float acc[4][8];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
#pragma unroll 4
    for (int m = 0; m < 32; ++m) {
        const float4 x = *reinterpret_cast<const float4 *>(P1 + m * 32 + r0);
        const float4 y0 = *reinterpret_cast<const float4 *>(P2 + m * 32 + c0);
        const float4 y1 = *reinterpret_cast<const float4 *>(P2 + m * 32 + c0 + 4);
        const float xv[4] = {x.x, x.y, x.z, x.w};
        const float yv[8] = {y0.x, y0.y, y0.z, y0.w, y1.x, y1.y, y1.z, y1.w};
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(xv[a], yv[b], acc[a][b]);
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
        float4 *cp = reinterpret_cast<float4 *>(C + (c0 + b) * 32 + r0);
        float4 v = *cp;
        v.x -= acc[0][b]; v.y -= acc[1][b]; v.z -= acc[2][b]; v.w -= acc[3][b];
        *cp = v;
    }
}

// step (a) for block row j by one warp of its owner: factor (L_jj stays in its
// slot), inverse into this CTA's xd area and to every CTA's inv buffer; on
// failure the first bad row is published to every CTA.  Nothing goes to global
// memory here: the write-out after the sweep does that.
LNB_DEV void pc_diag_step(cg::cluster_group &cl, int nb, int j, int64_t row0, float *own, float *inv, float *xd,
                          float *rv, int *s_fail, lnb_status_t *st, int q, int lane)
{
    float *D = own + pc_slot(j, j, q) * PBK;
    const int bad = pc_factor_block(D, rv, lane);
    if (bad) {
        const int fail = j * 32 + bad;
        if (lane == 0) {
            atomicCAS(&st->info, 0, (int)(row0 + fail));
            for (int r = 0; r < PCS; ++r) *cl.map_shared_rank(s_fail, r) = fail;
        }
        return;
    }
    float x[32];
    pc_inverse(D, rv, lane, x);
    float *xl = xd + (j == q ? 0 : 32 * PXS) + lane * PXS;
#pragma unroll
    for (int t = 0; t < 8; ++t)
        *reinterpret_cast<float4 *>(xl + 4 * t) = make_float4(x[4 * t], x[4 * t + 1], x[4 * t + 2], x[4 * t + 3]);
    if (j + 1 < nb) {
        for (int r = 0; r < PCS; ++r) {
            float *di = cl.map_shared_rank(inv, r) + lane * PXS;
#pragma unroll
            for (int t = 0; t < 8; ++t)
                *reinterpret_cast<float4 *>(di + 4 * t) =
                    make_float4(x[4 * t], x[4 * t + 1], x[4 * t + 2], x[4 * t + 3]);
        }
    }
}

__global__ void __cluster_dims__(PCS, 1, 1) __launch_bounds__(PNT, 1)
    k_potrf_cluster(float *A, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st)
{
    extern __shared__ __align__(16) float pcs[];
    float *own = pcs;                     // owned blocks, column-major 32 x 32
    float *pb = own + POWN * PBK;         // panel column j: pb[i] = L_ij
    float *inv = pb + PNB * PBK;          // X_j: inv[m PXS + p] = X[p][m]
    float *xd = inv + 32 * PXS;           // inverses of this CTA's diagonal blocks (rows i1, i2), same layout
    float *rv = xd + 2 * 32 * PXS;        // 1 / L[c][c] of the block being factored
    int *s_fail = reinterpret_cast<int *>(rv + 32);
    cg::cluster_group cl = cg::this_cluster();
    const int q = (int)cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = bs / 32;
    const int i1 = q, i2 = 2 * PCS - 1 - q;
    const bool has1 = i1 < nb, has2 = i2 < nb;
    if (tid == 0) *s_fail = 0;
    {
        // owned blocks (i, k <= i) in slot order: row i1 first, then row i2
        const int n1 = has1 ? i1 + 1 : 0, n2 = has2 ? i2 + 1 : 0;
        for (int idx = tid; idx < (n1 + n2) * 256; idx += PNT) {
            const int s = idx >> 8, e = idx & 255, c = e >> 3, t = e & 7;
            const int i = s < n1 ? i1 : i2, k = s < n1 ? s : s - n1;
            cp_async16(own + s * PBK + c * 32 + 4 * t, A + (int64_t)(i * 32 + 4 * t) + (int64_t)(k * 32 + c) * lda,
                       true);
        }
        cp_async_commit();
        cp_async_wait<0>();
    }
    cl.sync();                            // every CTA runs before any remote access
    if (q == 0 && warp == 0) pc_diag_step(cl, nb, 0, row0, own, inv, xd, rv, s_fail, st, q, lane);
    cl.sync();
    for (int j = 0; j + 1 < nb; ++j) {
        if (*s_fail) break;               // the same value in every CTA after the barrier
        // (c) owned blocks below the diagonal: L_ij = A_ij X^T; warps 4 w4 .. 4 w4 + 3
        //     take column quarters of the w4-th such block
        {
            int ib0 = -1, ib1 = -1;
            if (has1 && i1 > j) ib0 = i1;
            if (has2 && i2 > j) { if (ib0 < 0) ib0 = i2; else ib1 = i2; }
            const int i = (warp >> 2) == 0 ? ib0 : ib1;
            if (i >= 0) {
                const float *Aij = own + pc_slot(i, j, q) * PBK;
                const int r0 = 4 * (lane & 7), p0 = 8 * (warp & 3) + 2 * (lane >> 3);
                float acc[4][2];
#pragma unroll
                for (int a = 0; a < 4; ++a) acc[a][0] = acc[a][1] = 0.f;
#pragma unroll 8
                for (int m = 0; m < 32; ++m) {
                    const float4 av = *reinterpret_cast<const float4 *>(Aij + m * 32 + r0);
                    const float2 xv = *reinterpret_cast<const float2 *>(inv + m * PXS + p0);
                    const float a4[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
                    for (int a = 0; a < 4; ++a) {
                        acc[a][0] = fmaf(a4[a], xv.x, acc[a][0]);
                        acc[a][1] = fmaf(a4[a], xv.y, acc[a][1]);
                    }
                }
                const float4 o0 = make_float4(acc[0][0], acc[1][0], acc[2][0], acc[3][0]);
                const float4 o1 = make_float4(acc[0][1], acc[1][1], acc[2][1], acc[3][1]);
                for (int r = 0; r < PCS; ++r) {
                    float *dp = cl.map_shared_rank(pb, r) + i * PBK;
                    *reinterpret_cast<float4 *>(dp + p0 * 32 + r0) = o0;
                    *reinterpret_cast<float4 *>(dp + (p0 + 1) * 32 + r0) = o1;
                }
                // L_ij replaces A_ij in its slot once the group's four warps have read A_ij
                asm volatile("bar.sync %0, 128;" ::"r"(1 + (warp >> 2)) : "memory");
                float *Lo = own + pc_slot(i, j, q) * PBK;
                *reinterpret_cast<float4 *>(Lo + p0 * 32 + r0) = o0;
                *reinterpret_cast<float4 *>(Lo + (p0 + 1) * 32 + r0) = o1;
            }
        }
        cl.sync();
        // (e) A_ik -= L_ij L_kj^T for owned i, j < k <= i; items ordered row i1
        //     then row i2, so (j + 1, j + 1) is item 0 where this CTA owns it
        {
            const int n1 = (has1 && i1 > j) ? i1 - j : 0, n2 = (has2 && i2 > j) ? i2 - j : 0;
            const bool diag_next = pc_owner(j + 1) == q;
            int it = warp, step = PNT / 32;
            if (diag_next) { it = warp == 0 ? 0 : warp; step = warp == 0 ? n1 + n2 : PNT / 32 - 1; }
            for (; it < n1 + n2; it += step) {
                const int i = it < n1 ? i1 : i2, k = j + 1 + (it < n1 ? it : it - n1);
                pc_update(own + pc_slot(i, k, q) * PBK, pb + i * PBK, pb + k * PBK, lane);
            }
            if (diag_next && warp == 0) {
                __syncwarp();
                pc_diag_step(cl, nb, j + 1, row0, own, inv, xd, rv, s_fail, st, q, lane);
            }
        }
        cl.sync();
    }
    // Write-out.  A cluster barrier is a release: it waits until the CTA's earlier
    // global stores are acknowledged, so the sweep keeps every finished block in
    // shared memory and they all leave here.  Blocks (i, k) with k < jf are final
    // (jf = the block of a failed pivot, nb without one); the others, like the
    // upper triangle of the tile, keep their values in global memory.  Inverses:
    // the factored diagonal blocks', identity from jf on.
    const int fail = *s_fail;
    const int jf = fail ? (fail - 1) / 32 : nb;
    for (int rr = 0; rr < 2; ++rr) {
        const int i = rr == 0 ? i1 : i2;
        if (i >= nb) continue;
        const int kend = i + 1 < jf ? i + 1 : jf;
        for (int idx = tid; idx < kend * 256; idx += PNT) {
            const int k = idx >> 8, e = idx & 255, c = e >> 3, r = 4 * (e & 7);
            const float4 v = *reinterpret_cast<const float4 *>(own + pc_slot(i, k, q) * PBK + c * 32 + r);
            float *g = A + (int64_t)(i * 32 + r) + (int64_t)(k * 32 + c) * lda;
            if (k < i) {
                *reinterpret_cast<float4 *>(g) = v;
            } else {
                if (r >= c) g[0] = v.x;
                if (r + 1 >= c) g[1] = v.y;
                if (r + 2 >= c) g[2] = v.z;
                if (r + 3 >= c) g[3] = v.w;
            }
        }
        // dinv block i, column-major: dinv[i 1024 + m 32 + p] = X[p][m]
        for (int idx = tid; idx < 256; idx += PNT) {
            const int m = idx >> 3, p = 4 * (idx & 7);
            float4 v;
            if (i < jf) {
                v = *reinterpret_cast<const float4 *>(xd + rr * 32 * PXS + m * PXS + p);
            } else {
                v.x = (p == m) ? 1.f : 0.f; v.y = (p + 1 == m) ? 1.f : 0.f;
                v.z = (p + 2 == m) ? 1.f : 0.f; v.w = (p + 3 == m) ? 1.f : 0.f;
            }
            *reinterpret_cast<float4 *>(dinv + (int64_t)i * PBK + m * 32 + p) = v;
        }
    }
}

}  // namespace lnb

using namespace lnb;

// one diagonal tile of order bs (bs % 32 == 0, bs <= 512) by one cluster launch;
// A and dinv 16-byte aligned, lda % 4 == 0 (cudaErrorInvalidValue otherwise)
extern "C" int lnb_k_potrf_cluster_f32(float *A, int64_t lda, int bs, int64_t row0, float *dinv, lnb_status_t *st,
                                       lnb_stream_t s)
{
    if (bs <= 0) return 0;
    if (bs % 32 || bs > 32 * PNB || (uintptr_t)A % 16 || lda % 4 || (uintptr_t)dinv % 16)
        return (int)cudaErrorInvalidValue;
    static int attr = 0;
    if (!attr) {
        const cudaError_t e = cudaFuncSetAttribute(k_potrf_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, PC_SMEM);
        if (e != cudaSuccess) return (int)e;
        attr = 1;
    }
    k_potrf_cluster<<<PCS, PNT, PC_SMEM, s>>>(A, lda, bs, row0, dinv, st);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
