// k_bfactor.cuh -- single-CTA right-looking Cholesky of a matrix of order <= 512
// held in global memory (L2-resident): 32-column panels staged in shared memory
// by cp.async; warp 0 factors each diagonal block left-looking (potf2 order)
// while warp 1 inverts it one row behind; the rows below become dot products
// with that inverse; the trailing update runs 4 x 4 tiles per thread with
// 16-byte loads.  Also the triangular solves with the stored block inverses.
// Used per system by the batched solver (k_batched.cu) and per diagonal block
// by the block-Jacobi preconditioner of the sparse refinement (k_sparse.cu).
#pragma once
#include "common.cuh"

namespace lnb {

constexpr int BMAXN = 512, BP = 32;
constexpr int BMAXR = 8;                  // right-hand sides of one system
constexpr int BLDP = BMAXN + 4;           // stride of a staged panel column in shared memory

// 16-byte cp.async from L2 copying `bytes` (0..16) and zero-filling the rest
LNB_DEV void bcp16(void *smem, const void *gmem, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(bytes));
}

// sum_{p<len} a[p*sa] b[p*sb] with 8 loads of each operand in flight per step
template <typename T>
LNB_DEV T bdot(const T *a, int sa, const T *b, int sb, int len)
{
    T s0 = T(0), s1 = T(0), s2 = T(0), s3 = T(0);
    int p = 0;
    for (; p + 8 <= len; p += 8) {
        T x[8], y[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) { x[e] = a[(p + e) * sa]; y[e] = b[(p + e) * sb]; }
        s0 = fma(x[0], y[0], s0); s1 = fma(x[1], y[1], s1); s2 = fma(x[2], y[2], s2); s3 = fma(x[3], y[3], s3);
        s0 = fma(x[4], y[4], s0); s1 = fma(x[5], y[5], s1); s2 = fma(x[6], y[6], s2); s3 = fma(x[7], y[7], s3);
    }
    for (; p < len; ++p) s0 = fma(a[p * sa], b[p * sb], s0);
    return (s0 + s1) + (s2 + s3);
}
LNB_DEV float brsqrt(float x) { return rsqrtf(x); }
LNB_DEV double brsqrt(double x) { return rsqrt(x); }

template <int NT>
LNB_DEV double bmax_block(double v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < NT / 32; ++w) m = fmax(m, red[w]);
    __syncthreads();
    return m;
}

// 4-element vector load/store of TF from 16-byte-aligned memory (FP32: one
// float4; FP64: two double2)
LNB_DEV void ld4(const float *p, float (&v)[4])
{
    const float4 q = *reinterpret_cast<const float4 *>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
LNB_DEV void ld4(const double *p, double (&v)[4])
{
    const double2 q0 = *reinterpret_cast<const double2 *>(p), q1 = *reinterpret_cast<const double2 *>(p + 2);
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}
LNB_DEV void ld4cg(const float *p, float (&v)[4])
{
    const float4 q = __ldcg(reinterpret_cast<const float4 *>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
LNB_DEV void ld4cg(const double *p, double (&v)[4])
{
    const double2 q0 = __ldcg(reinterpret_cast<const double2 *>(p)), q1 = __ldcg(reinterpret_cast<const double2 *>(p + 2));
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}

// Right-looking Cholesky of the n x n matrix in F (lower, ld ldF, 16-byte
// aligned columns; rows up to n rounded up to 4 must be addressable), 32-column
// panels staged in shared memory.  Writes the 32 x 32 inverses of the diagonal
// blocks to Dv, column-major (Dk[r + 32 c] = inv[r][c]).  Returns info (0 or
// the 1-based first bad pivot), the same in every thread; after a failure the
// blocks from the failing one on are not written.
template <typename TF, int NT>
__device__ int bfactor(TF *F, int ldF, int n, TF *Dv, TF *P, TF *Li, TF *Rd, int *s_fail)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int V = 16 / (int)sizeof(TF);              // elements per 16-byte copy
    if (tid == 0) *s_fail = 0;
    for (int j0 = 0; j0 < n; j0 += BP) {
        const int jb = min(BP, n - j0), mr = n - j0;
        // stage P[c][r] = F[(j0 + r) + (j0 + c) ldF], r < mr, c < jb
        const int nch = (mr + V - 1) / V;
        for (int idx = tid; idx < jb * nch; idx += NT) {
            const int c = idx / nch, r = (idx - c * nch) * V;
            const int nv = min(V, mr - r);
            bcp16(P + c * BLDP + r, F + (j0 + r) + (int64_t)(j0 + c) * ldF, nv * (int)sizeof(TF));
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        // Diagonal block: warp 0 factors it column by column while warp 1 forms its
        // inverse one row behind.  Row r of the inverse needs row r of L and
        // 1/L[r][r], which factor step r completes, so the two warps meet at named
        // barrier 1 once per column (bar.sync on both sides: exactly 32 + 32
        // arrivals per generation).  A bad pivot at column c is recorded in
        // *s_fail (= j0 + c + 1) before barrier c; warp 0 leaves after barrier c
        // and warp 1 after the barrier at which it reads that value for its own
        // row c, so each has passed c + 1 barriers.
        if (warp == 0) {
            // left-looking (potf2 order); lane l owns row l
            const int rl = lane < jb ? lane : 0;
            for (int c = 0; c < jb; ++c) {
                const TF sv = P[c * BLDP + rl] - bdot(P + rl, BLDP, P + c, BLDP, c);
                const TF d = __shfl_sync(0xffffffffu, sv, c);
                const bool bad = !(d > TF(0));                  // warp-uniform: d is broadcast
                if (bad) {
                    if (lane == 0) *s_fail = j0 + c + 1;
                } else {
                    const TF inv = brsqrt(d);
                    if (lane == c) { P[c * BLDP + c] = d * inv; Rd[c] = inv; }
                    else if (lane > c && lane < jb) P[c * BLDP + lane] = sv * inv;
                }
                asm volatile("bar.sync 1, 64;" ::: "memory");   // column c published
                if (bad) break;
            }
        } else if (warp == 1) {
            // inverse of the block: lane c builds column c, Li[c][*] = inv[*][c]
            TF *Xc = Li + lane * (BP + 1);
            bool ok = true;
            for (int r = 0; r < BP; ++r) {
                TF v = (r == lane) ? TF(1) : TF(0);
                if (r < jb) {
                    asm volatile("bar.sync 1, 64;" ::: "memory");   // factor column r done
                    // warp 0 may already be one column ahead (and may have recorded a
                    // failure there), so only a failure AT column r ends this loop
                    if (*(volatile int *)s_fail == j0 + r + 1) { ok = false; break; }
                    v = (v - bdot(P + r, BLDP, Xc, 1, r)) * Rd[r];
                }
                Xc[r] = v;
            }
            if (ok) {
                __syncwarp();
                TF *Dk = Dv + (int64_t)(j0 / BP) * BP * BP;     // column-major: Dk[r + 32 c] = inv[r][c]
                for (int c = 0; c < BP; ++c) Dk[lane + BP * c] = Li[c * (BP + 1) + lane];
            }
        }
        __syncthreads();
        if (*s_fail) break;
        // rows below the block: x_r = b_r inv^T, 4 threads per row
        const int g = tid & 3;
        for (int rb = jb; rb < mr; rb += NT / 4) {
            const int r = rb + (tid >> 2);
            const bool act = r < mr;
            TF bv[BP];
#pragma unroll
            for (int p = 0; p < BP; ++p) bv[p] = (act && p < jb) ? P[p * BLDP + r] : TF(0);
            __syncwarp();
#pragma unroll
            for (int s = 0; s < BP / 4; ++s) {
                const int j = g + 4 * s;
                TF acc = TF(0);
#pragma unroll
                for (int p = 0; p < BP; ++p) acc = fma(bv[p], Li[p * (BP + 1) + j], acc);
                if (act && j < jb) P[j * BLDP + r] = acc;
            }
        }
        __syncthreads();
        // the finished panel back to F (16-byte runs; rows above the diagonal get
        // unused values)
        for (int idx = tid; idx < jb * nch; idx += NT) {
            const int c = idx / nch, r = (idx - c * nch) * V;
            TF *dst = F + (j0 + r) + (int64_t)(j0 + c) * ldF;
            if (r + V <= mr) {
                if constexpr (V == 4) *reinterpret_cast<float4 *>(dst) = *reinterpret_cast<const float4 *>(P + c * BLDP + r);
                else *reinterpret_cast<double2 *>(dst) = *reinterpret_cast<const double2 *>(P + c * BLDP + r);
            } else {
                for (int e = 0; r + e < mr; ++e) dst[e] = P[c * BLDP + r + e];
            }
        }
        // trailing update F[r][c] -= sum_p P[p][r] P[p][c], jb <= c <= r < mr (relative), 4x4 per thread
        const int tr = mr - jb;
        if (tr > 0) {
            const int nb4 = (tr + 3) / 4, nblk = nb4 * (nb4 + 1) / 2;
            for (int id = tid; id < nblk; id += NT) {
                int bi = (int)((sqrtf(8.0f * id + 1.0f) - 1.0f) * 0.5f);
                while (bi * (bi + 1) / 2 > id) --bi;
                while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
                const int bj = id - bi * (bi + 1) / 2;
                const int ra = jb + 4 * bi, rc = jb + 4 * bj;
                // C tile first (its loads overlap the products below)
                TF cv[4][4];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    if (rc + jj < mr) ld4cg(F + (j0 + ra) + (int64_t)(j0 + rc + jj) * ldF, cv[jj]);
                    else cv[jj][0] = cv[jj][1] = cv[jj][2] = cv[jj][3] = TF(0);
                }
                TF acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int jj = 0; jj < 4; ++jj) acc[i][jj] = TF(0);
#pragma unroll 8
                for (int p = 0; p < BP; ++p) {
                    TF av[4], cvv[4];
                    ld4(P + p * BLDP + ra, av);
                    ld4(P + p * BLDP + rc, cvv);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fma(av[i], cvv[jj], acc[i][jj]);
                }
#pragma unroll
                for (int jj = 0; jj < 4; ++jj) {
                    const int c = rc + jj;
                    if (c >= mr) continue;
                    TF *col = F + (j0 + ra) + (int64_t)(j0 + c) * ldF;
                    if (bi != bj && ra + 4 <= mr) {
                        TF o[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) o[i] = cv[jj][i] - acc[i][jj];
                        if constexpr (V == 4) *reinterpret_cast<float4 *>(col) = make_float4(o[0], o[1], o[2], o[3]);
                        else {
                            *reinterpret_cast<double2 *>(col) = make_double2(o[0], o[1]);
                            *reinterpret_cast<double2 *>(col + 2) = make_double2(o[2], o[3]);
                        }
                    } else {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (ra + i < mr && ra + i >= c) col[i] = cv[jj][i] - acc[i][jj];
                    }
                }
            }
        }
        __syncthreads();
    }
    return *s_fail;
}

// column stride of a 32 x 32 block inverse staged in shared memory: a multiple
// of 16 bytes (cp.async destinations) that spreads a row of the block over the
// banks (at most 4-way conflicts when the lanes walk a row)
template <typename TF>
__host__ __device__ constexpr int bsd_ld() { return sizeof(TF) == 4 ? BP + 4 : BP + 2; }
template <typename TF>
__host__ __device__ constexpr int bsd_bytes() { return (int)sizeof(TF) * BP * bsd_ld<TF>(); }

// start the copy of one block inverse (column-major, 32 x 32) into sD
// (column stride bsd_ld); the caller waits with cp_async_wait<0> + a barrier
template <typename TF, int NT>
LNB_DEV void bstage_inv(TF *sD, const TF *Dk)
{
    constexpr int CPC = BP * (int)sizeof(TF) / 16;           // 16-byte chunks per column
    for (int i = threadIdx.x; i < BP * CPC; i += NT) {
        const int c = i / CPC, o = i - c * CPC;
        bcp16(sD + c * bsd_ld<TF>() + o * (16 / (int)sizeof(TF)), Dk + c * BP + o * (16 / (int)sizeof(TF)), 16);
    }
    cp_async_commit();
}

// z <- inv(L) z, then z <- inv(L^T) z, for nr columns of z in shared memory
// (z[q * BMAXN + i]); L in F, the block inverses in Dv.  env (may be NULL):
// the factor's envelope per 32-row tile t -- env[t] = the first column with a
// nonzero in rows 32t .. 32t+31, env[BMAXN/BP + t] = the last row with a
// nonzero in columns 32t .. 32t+31 -- so the sums skip tiles that are zero.
// sD: bsd_bytes<TF>() of shared memory.  Each block's inverse is copied there
// by cp.async while the block's partial sums run, so the block step reads it
// from shared memory instead of waiting on one L2 load per term.
template <typename TF, int NT>
__device__ void bsolve(const TF *F, int ldF, const TF *Dv, int n, int nr, double *z, double *red, TF *sD,
                       const int *env = nullptr)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    static_assert(BMAXR <= NW, "one warp per right-hand side in the block-inverse steps");
    const int nblk = (n + BP - 1) / BP;
    // forward
    for (int kb = 0; kb < nblk; ++kb) {
        const int k0 = kb * BP, kn = min(BP, n - k0);
        const int cs = env ? env[kb] : 0;                   // columns before cs are zero in these rows
        const TF *Dk = Dv + (int64_t)kb * BP * BP;
        bstage_inv<TF, NT>(sD, Dk);
        if (k0 > cs) {
            double acc[BMAXR];
#pragma unroll
            for (int q = 0; q < BMAXR; ++q) acc[q] = 0.0;
            if (lane < kn) {
#pragma unroll 4
                for (int c = cs + warp; c < k0; c += NW) {
                    const double f = (double)__ldcg(F + (k0 + lane) + (int64_t)c * ldF);
#pragma unroll
                    for (int q = 0; q < BMAXR; ++q)
                        if (q < nr) acc[q] = fma(f, z[q * BMAXN + c], acc[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < BMAXR; ++q) red[(q * NW + warp) * BP + lane] = acc[q];   // lanes contiguous
            cp_async_wait<0>();
            __syncthreads();
            for (int t = tid; t < kn * nr; t += NT) {
                const int q = t / kn, i = t - q * kn;
                double s = 0.0;
                for (int w = 0; w < NW; ++w) s += red[(q * NW + w) * BP + i];
                z[q * BMAXN + k0 + i] -= s;
            }
            __syncthreads();
        } else {
            cp_async_wait<0>();
            __syncthreads();
        }
        // z_blk = inv(L_kk) z_blk: thread (j, q), j = row of the block, q = rhs
        const int j = tid & 31, q = tid >> 5;
        const bool act = j < kn && q < nr;
        double v = 0.0;
        if (act)
            for (int p = 0; p <= j; ++p) v = fma((double)sD[j + bsd_ld<TF>() * p], z[q * BMAXN + k0 + p], v);
        __syncthreads();
        if (act) z[q * BMAXN + k0 + j] = v;
        __syncthreads();
    }
    // backward
    for (int kb = nblk - 1; kb >= 0; --kb) {
        const int k0 = kb * BP, kn = min(BP, n - k0), r0 = k0 + kn;
        const int re = env ? min(n, env[BMAXN / BP + kb] + 1) : n;    // rows from re on are zero here
        bstage_inv<TF, NT>(sD, Dv + (int64_t)kb * BP * BP);
        if (r0 < re) {
            for (int jc = warp; jc < kn; jc += NW) {
                double acc[BMAXR];
#pragma unroll
                for (int q = 0; q < BMAXR; ++q) acc[q] = 0.0;
                const TF *col = F + (int64_t)(k0 + jc) * ldF;
#pragma unroll 4
                for (int r = r0 + lane; r < re; r += 32) {
                    const double f = (double)__ldcg(col + r);
#pragma unroll
                    for (int q = 0; q < BMAXR; ++q)
                        if (q < nr) acc[q] = fma(f, z[q * BMAXN + r], acc[q]);
                }
#pragma unroll
                for (int q = 0; q < BMAXR; ++q) {
                    double v = acc[q];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                    if (lane == 0) red[q * BP + jc] = v;
                }
            }
            cp_async_wait<0>();
            __syncthreads();
            for (int t = tid; t < kn * nr; t += NT) {
                const int q = t / kn, i = t - q * kn;
                z[q * BMAXN + k0 + i] -= red[q * BP + i];
            }
            __syncthreads();
        } else {
            cp_async_wait<0>();
            __syncthreads();
        }
        // z_blk = inv(L_kk)^T z_blk
        const int j = tid & 31, q = tid >> 5;
        const bool act = j < kn && q < nr;
        double v = 0.0;
        if (act)
            for (int p = j; p < kn; ++p) v = fma((double)sD[p + bsd_ld<TF>() * j], z[q * BMAXN + k0 + p], v);
        __syncthreads();
        if (act) z[q * BMAXN + k0 + j] = v;
        __syncthreads();
    }
}

}  // namespace lnb
