// k_batched.cu -- many independent uneven SPD systems in one persistent launch.
//
// Each system is the reference's SPD solve (dspdsolv_main, spdsolv_main.c:10-20:
// tile Cholesky then the forward and backward solves) followed, in the
// low-precision mode, by the refinement of itref.c (FP64 residual and
// update).  A CTA takes systems from an atomic ticket over a cost-sorted
// order (largest first), so the uneven sizes balance over the SMs; the whole
// batch is one launch and can be captured in a CUDA graph.
//
// Per system (n <= 512, nrhs <= 8), in one CTA of BT threads:
//   1. the lower triangle of A (FP64) is copied into the CTA's scratch factor
//      F (type TF = float or double, ld n; L2-resident)
//   2. right-looking Cholesky with PW-wide panels: the panel is staged in
//      shared memory, warp 0 factors its diagonal block with shuffles, all
//      threads solve the rows below and apply the rank-PW update to F
//   3. x = 0, r = b; repeat: z = F^-T F^-1 r (blocked by PW rows), x += z,
//      r = b - A x in FP64 from the original A; stop at backward error
//      ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol, at most max_iter
//      times (one pass, no refinement, when TF = double)
#include "common.cuh"

namespace lnb {

constexpr int BMAXN = 512, BMAXR = 8;

struct BatchArgs {
    int count;
    const int *n, *nrhs;
    const int64_t *a_off, *b_off;
    const double *A, *B;
    double *X;
    void *scratch;            // per-CTA factor scratch: BMAXN * BMAXN elements each
    const int *order;         // processing order (cost-sorted)
    int *ticket;
    int *info, *iters;
    int max_iter;
    double tol_eps;           // tol = tol_eps * n
};

template <typename TF, int PW>
__device__ int factor_one(TF *F, int n, const double *A, TF *Ps)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    __shared__ int fail;
    if (tid == 0) fail = 0;
    // lower triangle of A into F
    for (int idx = tid; idx < n * n; idx += nt) {
        const int c = idx / n, r = idx - c * n;
        if (r >= c) F[r + c * n] = (TF)A[r + (int64_t)c * n];
    }
    __syncthreads();
    constexpr int LDP = PW + 1;
    for (int j0 = 0; j0 < n; j0 += PW) {
        const int jb = min(PW, n - j0), mr = n - j0;
        // stage the panel rows j0..n, cols j0..j0+jb
        for (int idx = tid; idx < mr * jb; idx += nt) {
            const int c = idx / mr, r = idx - c * mr;
            Ps[r * LDP + c] = F[(j0 + r) + (j0 + c) * n];
        }
        __syncthreads();
        if (warp == 0) {
            TF x[PW];
#pragma unroll
            for (int c = 0; c < PW; ++c) x[c] = (lane < jb && c < jb && lane >= c) ? Ps[lane * LDP + c] : TF(0);
            int bad = 0;
#pragma unroll
            for (int c = 0; c < PW; ++c) {
                if (c < jb && !bad) {
                    const TF d = __shfl_sync(0xffffffffu, x[c], c);
                    if (!(d > TF(0))) {
                        bad = j0 + c + 1;
                    } else {
                        const TF dd = sqrt(d);
                        if (lane == c) x[c] = dd;
                        else if (lane > c) x[c] = x[c] / dd;
#pragma unroll
                        for (int cc = c + 1; cc < PW; ++cc) {
                            const TF l = __shfl_sync(0xffffffffu, x[c], cc);
                            if (lane >= cc) x[cc] -= x[c] * l;
                        }
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < PW; ++c)
                if (lane < jb && c < jb && lane >= c) Ps[lane * LDP + c] = x[c];
            if (lane == 0 && bad) fail = bad;
        }
        __syncthreads();
        if (fail) break;
        for (int r = jb + tid; r < mr; r += nt) {
            TF x[PW];
#pragma unroll
            for (int c = 0; c < PW; ++c) {
                if (c < jb) {
                    TF v = Ps[r * LDP + c];
#pragma unroll
                    for (int p = 0; p < c; ++p) v -= x[p] * Ps[c * LDP + p];
                    x[c] = v / Ps[c * LDP + c];
                    Ps[r * LDP + c] = x[c];
                }
            }
        }
        __syncthreads();
        for (int idx = tid; idx < mr * jb; idx += nt) {
            const int c = idx / mr, r = idx - c * mr;
            if (r >= c) F[(j0 + r) + (j0 + c) * n] = Ps[r * LDP + c];
        }
        // trailing update of F (lower), 4x4 blocks per thread; loads before stores
        const int t0 = jb, tr = mr - jb;
        if (tr > 0) {
            const int nb4 = (tr + 3) / 4, nblk = nb4 * (nb4 + 1) / 2;
            for (int id = tid; id < nblk; id += nt) {
                int bi = (int)((sqrtf(8.0f * id + 1.0f) - 1.0f) * 0.5f);
                while (bi * (bi + 1) / 2 > id) --bi;
                while ((bi + 1) * (bi + 2) / 2 <= id) ++bi;
                const int bj = id - bi * (bi + 1) / 2;
                const int ra = t0 + 4 * bi, rb = t0 + 4 * bj;
                TF acc[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = TF(0);
                for (int p = 0; p < jb; ++p) {
                    TF a[4], bb[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        a[i] = (ra + i < mr) ? Ps[(ra + i) * LDP + p] : TF(0);
                        bb[i] = (rb + i < mr) ? Ps[(rb + i) * LDP + p] : TF(0);
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
                }
                TF cv[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int r = ra + i, c = rb + j;
                        cv[i][j] = (r < mr && c < mr && r >= c) ? F[(j0 + r) + (j0 + c) * n] : TF(0);
                    }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int r = ra + i, c = rb + j;
                        if (r < mr && c < mr && r >= c) F[(j0 + r) + (j0 + c) * n] = cv[i][j] - acc[i][j];
                    }
            }
        }
        __syncthreads();
    }
    __syncthreads();
    return fail;   // block-uniform: every thread reads the shared flag after the barrier
}

// z <- F^-T F^-1 z in place (z: n x nr doubles in shared memory, ld BMAXN).
// Blocked by PW rows: the off-diagonal part of each block row is a sum split
// over all threads (reduced in shared memory), the PW x PW triangle is one
// thread per right-hand side.
template <typename TF, int PW>
__device__ void solve_one(const TF *F, int n, int nr, double *z, double *red)
{
    const int tid = threadIdx.x, nt = blockDim.x, nparts = nt / PW;
    for (int k0 = 0; k0 < n; k0 += PW) {              // forward: z_k -= L_k,0:k z_0:k
        const int kb = min(PW, n - k0);
        for (int q = 0; q < nr; ++q) {
            const int i = tid % PW, part = tid / PW;
            double s = 0.0;
            if (i < kb)
                for (int j = part; j < k0; j += nparts) s += (double)F[(k0 + i) + j * n] * z[j + q * BMAXN];
            red[part * PW + i] = s;
            __syncthreads();
            if (tid < kb) {
                double t = 0.0;
                for (int p = 0; p < nparts; ++p) t += red[p * PW + tid];
                z[(k0 + tid) + q * BMAXN] -= t;
            }
            __syncthreads();
        }
        if (tid < nr) {
            const int q = tid;
            for (int i = 0; i < kb; ++i) {
                double s = z[(k0 + i) + q * BMAXN];
                for (int j = 0; j < i; ++j) s -= (double)F[(k0 + i) + (k0 + j) * n] * z[(k0 + j) + q * BMAXN];
                z[(k0 + i) + q * BMAXN] = s / (double)F[(k0 + i) + (k0 + i) * n];
            }
        }
        __syncthreads();
    }
    for (int k0 = ((n - 1) / PW) * PW; k0 >= 0; k0 -= PW) {   // backward: z_k -= L_{k+1:,k}^T z_{k+1:}
        const int kb = min(PW, n - k0);
        for (int q = 0; q < nr; ++q) {
            const int part = tid % nparts, i = tid / nparts;   // consecutive threads -> consecutive j
            double s = 0.0;
            if (i < kb)
                for (int j = k0 + kb + part; j < n; j += nparts) s += (double)F[j + (k0 + i) * n] * z[j + q * BMAXN];
            red[part * PW + i] = s;
            __syncthreads();
            if (tid < kb) {
                double t = 0.0;
                for (int p = 0; p < nparts; ++p) t += red[p * PW + tid];
                z[(k0 + tid) + q * BMAXN] -= t;
            }
            __syncthreads();
        }
        if (tid < nr) {
            const int q = tid;
            for (int i = kb - 1; i >= 0; --i) {
                double s = z[(k0 + i) + q * BMAXN];
                for (int j = i + 1; j < kb; ++j) s -= (double)F[(k0 + j) + (k0 + i) * n] * z[(k0 + j) + q * BMAXN];
                z[(k0 + i) + q * BMAXN] = s / (double)F[(k0 + i) + (k0 + i) * n];
            }
        }
        __syncthreads();
    }
}

LNB_DEV double block_max(double v, double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < nw; ++w) m = fmax(m, red[w]);
    __syncthreads();
    return m;
}

template <typename TF, int PW>
__global__ void __launch_bounds__(256) k_batched_posv(BatchArgs a)
{
    extern __shared__ __align__(16) unsigned char smb[];
    double *x = (double *)smb;                     // [BMAXR][BMAXN]
    double *r = x + BMAXR * BMAXN;                 // [BMAXR][BMAXN]
    TF *Ps = (TF *)(r + BMAXR * BMAXN);            // panel [BMAXN][PW+1]
    __shared__ double red[256];
    __shared__ int s_item;
    TF *F = (TF *)a.scratch + (int64_t)blockIdx.x * BMAXN * BMAXN;
    const int tid = threadIdx.x, nt = blockDim.x;
    while (true) {
        if (tid == 0) s_item = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= a.count) break;
        const int sys = a.order ? a.order[item] : item;
        const int n = a.n[sys], nr = a.nrhs[sys];
        if (n < 1 || n > BMAXN || nr < 1 || nr > BMAXR) {   // outside the kernel's fixed capacity
            if (tid == 0) {
                if (a.info) a.info[sys] = -7;
                if (a.iters) a.iters[sys] = 0;
            }
            __syncthreads();
            continue;
        }
        const double *A = a.A + a.a_off[sys];
        const double *B = a.B + a.b_off[sys];
        double *Xo = a.X + a.b_off[sys];
        const int info = factor_one<TF, PW>(F, n, A, Ps);   // same value in every thread
        __syncthreads();
        int it = 0;
        if (info == 0) {
            // ||A||_inf (full symmetric storage) and ||b||_inf per rhs
            double amax = 0.0;
            for (int i = tid; i < n; i += nt) {
                double s = 0.0;
                for (int j = 0; j < n; ++j) s += fabs(A[i + (int64_t)j * n]);
                amax = fmax(amax, s);
            }
            const double anorm = block_max(amax, red);
            for (int idx = tid; idx < BMAXR * BMAXN; idx += nt) x[idx] = 0.0;
            for (int idx = tid; idx < n * nr; idx += nt) {
                const int i = idx % n, q = idx / n;
                r[i + q * BMAXN] = B[i + (int64_t)q * n];
            }
            __syncthreads();
            const double tol = a.tol_eps * n;
            const int maxit = (sizeof(TF) == 8) ? 1 : a.max_iter;
            for (it = 1; it <= maxit; ++it) {
                solve_one<TF, PW>(F, n, nr, r, red);                  // r <- M^-1 r
                for (int idx = tid; idx < n * nr; idx += nt) {
                    const int i = idx % n, q = idx / n;
                    x[i + q * BMAXN] += r[i + q * BMAXN];
                }
                __syncthreads();
                // r = b - A x  (FP64), with ||r||, ||x||, ||b|| per rhs
                double worst = 0.0;
                for (int q = 0; q < nr; ++q) {
                    double rm = 0.0, xm = 0.0, bm = 0.0;
                    for (int i = tid; i < n; i += nt) {
                        double s = B[i + (int64_t)q * n];
                        bm = fmax(bm, fabs(s));
                        for (int j = 0; j < n; ++j) s -= A[i + (int64_t)j * n] * x[j + q * BMAXN];
                        r[i + q * BMAXN] = s;
                        rm = fmax(rm, fabs(s));
                        xm = fmax(xm, fabs(x[i + q * BMAXN]));
                    }
                    rm = block_max(rm, red);
                    xm = block_max(xm, red);
                    bm = block_max(bm, red);
                    const double den = anorm * xm + bm;
                    const double be = den > 0.0 ? rm / den : 0.0;
                    worst = fmax(worst, be);
                }
                if (worst <= tol) break;
            }
            if (it > maxit) it = maxit;
            for (int idx = tid; idx < n * nr; idx += nt) {
                const int i = idx % n, q = idx / n;
                Xo[i + (int64_t)q * n] = x[i + q * BMAXN];
            }
        }
        if (tid == 0) {
            if (a.info) a.info[sys] = info;
            if (a.iters) a.iters[sys] = it;
        }
        __syncthreads();
    }
}

// processing order: systems by decreasing n (a counting sort; one CTA)
__global__ void __launch_bounds__(1024) k_batch_order(int count, const int *n, int *order)
{
    __shared__ int hist[BMAXN + 2];
    for (int i = threadIdx.x; i < BMAXN + 2; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < count; s += blockDim.x) {
        int v = n[s];
        v = v < 0 ? 0 : (v > BMAXN ? BMAXN + 1 : v);
        atomicAdd(&hist[v], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {      // start offset of each size, largest size first
        int acc = 0;
        for (int v = BMAXN + 1; v >= 0; --v) {
            const int c = hist[v];
            hist[v] = acc;
            acc += c;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < count; s += blockDim.x) {
        int v = n[s];
        v = v < 0 ? 0 : (v > BMAXN ? BMAXN + 1 : v);
        order[atomicAdd(&hist[v], 1)] = s;
    }
}

}  // namespace lnb

using namespace lnb;

extern "C" int lnb_k_batch_order(int count, const int *n, int *order, lnb_stream_t s)
{
    k_batch_order<<<1, 1024, 0, s>>>(count, n, order);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" size_t lnb_batched_scratch_bytes(int grid, int fp64)
{
    return (size_t)grid * BMAXN * BMAXN * (fp64 ? 8 : 4);
}

extern "C" int lnb_k_batched_posv(int count, const int *n, const int *nrhs, const int64_t *a_off,
                                  const int64_t *b_off, const double *A, const double *B, double *X, void *scratch,
                                  int grid, const int *order, int *ticket, int *info, int *iters, int max_iter,
                                  int fp64, int pw, lnb_stream_t s)
{
    BatchArgs a;
    a.count = count; a.n = n; a.nrhs = nrhs; a.a_off = a_off; a.b_off = b_off; a.A = A; a.B = B; a.X = X;
    a.scratch = scratch; a.order = order; a.ticket = ticket; a.info = info; a.iters = iters;
    a.max_iter = max_iter; a.tol_eps = 10.0 * 1.1102230246251565e-16;
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(int), s);
    if (e != cudaSuccess) return (int)e;
    const size_t vec = 2 * BMAXR * BMAXN * sizeof(double);
    if (fp64) {
        if (pw == 32) {
            const int smem = (int)(vec + BMAXN * 33 * sizeof(double));
            cudaFuncSetAttribute(k_batched_posv<double, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            k_batched_posv<double, 32><<<grid, 256, smem, s>>>(a);
        } else {
            const int smem = (int)(vec + BMAXN * 17 * sizeof(double));
            cudaFuncSetAttribute(k_batched_posv<double, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            k_batched_posv<double, 16><<<grid, 256, smem, s>>>(a);
        }
    } else {
        if (pw == 32) {
            const int smem = (int)(vec + BMAXN * 33 * sizeof(float));
            cudaFuncSetAttribute(k_batched_posv<float, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            k_batched_posv<float, 32><<<grid, 256, smem, s>>>(a);
        } else {
            const int smem = (int)(vec + BMAXN * 17 * sizeof(float));
            cudaFuncSetAttribute(k_batched_posv<float, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            k_batched_posv<float, 16><<<grid, 256, smem, s>>>(a);
        }
    }
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
