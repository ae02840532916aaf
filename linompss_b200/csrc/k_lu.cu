// k_lu.cu -- kernels of the tile LU with partial pivoting (lu_main.c, the
// LAPACK dgetrf / dlaswp / dtrsm tasks of lu_kernels.c) and of the general
// solve (gensolv_main.c).
//
//   panel : factor the nb-wide panel A[c0:m, c0:c0+nb] (nb <= 32) in place with
//           partial pivoting, one thread-block cluster (1..8 CTAs).  CTA q
//           holds rows c0 + q R .. c0 + (q+1) R - 1 of the panel in shared
//           memory.  Per column k: each CTA finds its largest |a| at or below
//           row c0+k (ties: the smaller row, as idamax takes the first), the
//           CTAs read each other's candidates through distributed shared
//           memory, the owner of the pivot row broadcasts it into every CTA
//           (it becomes the U row), the owner of row c0+k hands the old row to
//           the pivot's owner, and every CTA scales its rows below by the
//           pivot and applies the rank-1 update.  Two cluster barriers per
//           column, no spin-waits.  Pivots are written LAPACK-style (1-based,
//           global row); an exactly zero pivot sets info (first one wins) and
//           skips the scaling, as dgetf2 does.
//   laswp : the panel's row swaps applied to other columns, one thread per
//           column, swaps in pivot order.
//   trsm  : X = L11^-1 X with L11 the panel's unit-lower nb x nb top block,
//           one thread per column of X.
#include <cooperative_groups.h>
#include <float.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace lnb {
namespace lu {

constexpr int NT = 256;
constexpr int MAXNB = 32;
constexpr int MAXCL = 8;
constexpr int SMEM_DATA = 200 * 1024;     // panel rows held by one CTA (one more row of rounding allowed)
constexpr int SMEM_MAX = SMEM_DATA + 4096;

__global__ void __launch_bounds__(NT) k_lu_panel(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int R,
                                                 int *piv, lnb_status_t *st)
{
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), ncl = (int)cl.num_blocks();
    extern __shared__ __align__(16) double psm[];
    double *P = psm;                      // P[j * R + r]: column j of my rows
    double *urow = P + (int64_t)nb * R;   // the pivot row (U row of this column), every CTA
    double *swp = urow + MAXNB;           // the old row k, at the pivot row's owner
    double *cand = swp + MAXNB;           // [0] = |max|, [1] = its global row
    __shared__ double wv[NT / 32];
    __shared__ long long wi[NT / 32];
    __shared__ long long s_p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t r0 = c0 + (int64_t)rank * R;
    const int nr = (int)(r0 < m ? (m - r0 < R ? m - r0 : R) : 0);

    for (int64_t i = tid; i < (int64_t)nb * R; i += NT) {
        const int j = (int)(i / R), r = (int)(i % R);
        P[i] = r < nr ? A[(r0 + r) + (c0 + j) * lda] : 0.0;
    }
    __syncthreads();

    for (int k = 0; k < nb; ++k) {
        const int64_t gk = c0 + k;
        // 1. my candidate
        double best = -1.0;
        long long bi = LLONG_MAX;
        for (int r = tid; r < nr; r += NT) {
            const int64_t g = r0 + r;
            if (g < gk) continue;
            const double v = fabs(P[(int64_t)k * R + r]);
            if (v > best) { best = v; bi = g; }          // rows visited in increasing order per thread
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const long long oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { wv[warp] = best; wi[warp] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < NT / 32; ++w)
                if (wv[w] > best || (wv[w] == best && wi[w] < bi)) { best = wv[w]; bi = wi[w]; }
            cand[0] = best;                                  // -1: no row of mine at or below c0+k
            cand[1] = bi == LLONG_MAX ? -1.0 : (double)bi;
        }
        if (ncl > 1) cl.sync(); else __syncthreads();          // #1: candidates visible
        // 2. the pivot row, the same in every CTA: lane q of warp 0 reads CTA q's candidate
        if (warp == 0) {
            double gb = -1.0;
            long long gi = LLONG_MAX;
            if (lane < ncl) {
                const double *cq = cl.map_shared_rank(cand, lane);
                if (cq[1] >= 0.0) { gb = cq[0]; gi = (long long)cq[1]; }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {                  // ncl <= 8
                const double ov = __shfl_down_sync(0xffffffffu, gb, o);
                const long long oi = __shfl_down_sync(0xffffffffu, gi, o);
                if (ov > gb || (ov == gb && oi < gi)) { gb = ov; gi = oi; }
            }
            if (lane == 0) s_p = gi;
        }
        __syncthreads();
        const int64_t p = s_p;
        const int ok = (int)((gk - c0) / R), op = (int)((p - c0) / R);
        // 3. exchange
        if (rank == op) {
            for (int i = tid; i < ncl * nb; i += NT) {
                const int q = i / nb, j = i % nb;
                double *uq = cl.map_shared_rank(urow, q);
                uq[j] = P[(int64_t)j * R + (p - r0)];
            }
        }
        if (rank == ok && p != gk) {
            double *sq = cl.map_shared_rank(swp, op);
            for (int j = tid; j < nb; j += NT) sq[j] = P[(int64_t)j * R + (gk - r0)];
        }
        if (ncl > 1) cl.sync(); else __syncthreads();          // #2: pivot row and old row delivered
        if (rank == ok)
            for (int j = tid; j < nb; j += NT) P[(int64_t)j * R + (gk - r0)] = urow[j];
        if (rank == op && p != gk)
            for (int j = tid; j < nb; j += NT) P[(int64_t)j * R + (p - r0)] = swp[j];
        __syncthreads();
        // 4. scale and rank-1 update of my rows below the pivot
        const double pv = urow[k];
        if (pv == 0.0 && rank == 0 && tid == 0) atomicCAS(&st->info, 0, (int)(gk + 1));
        for (int r = tid; r < nr; r += NT) {
            if (r0 + r <= gk) continue;
            double l = P[(int64_t)k * R + r];
            if (pv != 0.0) {
                l = l / pv;
                P[(int64_t)k * R + r] = l;
            }
            for (int j = k + 1; j < nb; ++j) P[(int64_t)j * R + r] -= l * urow[j];
        }
        if (rank == 0 && tid == 0) piv[gk] = (int)(p + 1);
        __syncthreads();
    }
    for (int64_t i = tid; i < (int64_t)nb * R; i += NT) {
        const int j = (int)(i / R), r = (int)(i % R);
        if (r < nr) A[(r0 + r) + (c0 + j) * lda] = P[i];
    }
    if (ncl > 1) cl.sync();                                  // no CTA leaves while its smem may be read
}

// rows k and piv[k]-1 swap, k = k0..k1-1 in order, on columns [a0, a1) and [b0, b1)
__global__ void k_laswp(double *A, int64_t lda, int64_t k0, int64_t k1, const int *piv, int64_t a0, int64_t a1,
                        int64_t b0, int64_t b1)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t na = a1 > a0 ? a1 - a0 : 0, nbb = b1 > b0 ? b1 - b0 : 0;
    if (t >= na + nbb) return;
    const int64_t j = t < na ? a0 + t : b0 + (t - na);
    double *col = A + j * lda;
    for (int64_t k = k0; k < k1; ++k) {
        const int64_t p = (int64_t)__ldg(piv + k) - 1;
        if (p != k) {
            const double x = col[k];
            col[k] = col[p];
            col[p] = x;
        }
    }
}

// X (rows c0 .. c0+nb-1, columns [j0, j1)) = L11^-1 X, L11 = A[c0:c0+nb, c0:c0+nb] unit lower
__global__ void __launch_bounds__(128) k_lu_trsm_unit(double *A, int64_t lda, int64_t c0, int nb, int64_t j0,
                                                      int64_t j1)
{
    __shared__ double L[MAXNB][MAXNB + 1];
    for (int i = threadIdx.x; i < nb * nb; i += blockDim.x) {
        const int r = i % nb, c = i / nb;
        L[r][c] = A[(c0 + r) + (c0 + c) * lda];
    }
    __syncthreads();
    const int64_t j = j0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= j1) return;
    double *x = A + c0 + j * lda;
    double v[MAXNB];
#pragma unroll
    for (int r = 0; r < MAXNB; ++r) v[r] = r < nb ? x[r] : 0.0;
#pragma unroll
    for (int r = 1; r < MAXNB; ++r) {
        double s = v[r];
#pragma unroll
        for (int c = 0; c < r; ++c) s -= L[r][c] * v[c];
        v[r] = s;
    }
#pragma unroll
    for (int r = 0; r < MAXNB; ++r)
        if (r < nb) x[r] = v[r];
}

}  // namespace lu
}  // namespace lnb

using namespace lnb::lu;

// Panel width for `rows` rows: the widest (<= 32, a power of two) whose rows
// fit a cluster of up to 8 CTAs; 0 if none fits.  Narrower panels that fit one
// CTA were measured slower on B200 (n = 1500: 11.5 vs 10.2 ms; n = 4096: 45.7
// vs 34.2 ms): the extra panels' launches cost more than the cluster barriers.
extern "C" int lnb_lu_panel_width(int64_t rows)
{
    for (int nb = MAXNB; nb >= 4; nb >>= 1)
        if (rows * nb * (int64_t)sizeof(double) <= (int64_t)MAXCL * SMEM_DATA) return nb;
    return 0;
}

extern "C" int lnb_k_lu_panel_f64(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int *piv, lnb_status_t *st,
                                  lnb_stream_t s)
{
    const int64_t rows = m - c0;
    if (rows <= 0 || nb <= 0) return 0;
    if (nb > MAXNB) return (int)cudaErrorInvalidValue;
    const int64_t bytes = rows * nb * (int64_t)sizeof(double);
    int ncl = (int)((bytes + SMEM_DATA - 1) / SMEM_DATA);
    if (ncl < 1) ncl = 1;
    if (ncl > MAXCL) return (int)cudaErrorInvalidValue;
    const int R = (int)((rows + ncl - 1) / ncl);
    const size_t smem = ((size_t)nb * R + 2 * MAXNB + 2) * sizeof(double);
    if (smem > (size_t)SMEM_MAX) return (int)cudaErrorInvalidValue;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_lu_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_MAX);
        if (e != cudaSuccess) return (int)e;
        e = cudaFuncSetAttribute(k_lu_panel, cudaFuncAttributeNonPortableClusterSizeAllowed, 0);
        if (e != cudaSuccess) return (int)e;
        attr = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ncl);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = (cudaStream_t)s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ncl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_lu_panel, A, lda, m, c0, nb, R, piv, st);
    lnb_prof_count(1);
    return (int)e;
}

extern "C" int lnb_k_laswp_f64(double *A, int64_t lda, int64_t k0, int64_t k1, const int *piv, int64_t a0,
                               int64_t a1, int64_t b0, int64_t b1, lnb_stream_t s)
{
    const int64_t ncols = (a1 > a0 ? a1 - a0 : 0) + (b1 > b0 ? b1 - b0 : 0);
    if (ncols <= 0 || k1 <= k0) return 0;
    k_laswp<<<(unsigned)((ncols + 127) / 128), 128, 0, (cudaStream_t)s>>>(A, lda, k0, k1, piv, a0, a1, b0, b1);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_lu_trsm_unit_f64(double *A, int64_t lda, int64_t c0, int nb, int64_t j0, int64_t j1,
                                      lnb_stream_t s)
{
    if (j1 <= j0 || nb <= 1) return 0;
    if (nb > MAXNB) return (int)cudaErrorInvalidValue;
    k_lu_trsm_unit<<<(unsigned)((j1 - j0 + 127) / 128), 128, 0, (cudaStream_t)s>>>(A, lda, c0, nb, j0, j1);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
