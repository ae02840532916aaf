// k_lu.cu -- kernels of the tile LU with partial pivoting (lu_main.c, the
// LAPACK dgetrf / dlaswp / dtrsm tasks of lu_kernels.c) and of the general
// solve (gensolv_main.c).
//
//   panel : factor the nb-wide panel A[c0:m, c0:c0+nb] (nb <= 32) in place with
//           partial pivoting, one thread-block cluster (1..8 CTAs of 512
//           threads), the panel held in registers (each thread 1..8 rows).
//           Per column k: each CTA finds its largest |a| at or below row c0+k
//           (ties: the smaller row, as idamax takes the first), the CTAs read
//           each other's candidates through distributed shared memory, the
//           pivot row (the U row) and the old row c0+k are exchanged through
//           the owners' shared memory, and every thread scales and updates
//           its rows below the pivot.  Two cluster barriers per column, no
//           spin-waits.  Pivots are written LAPACK-style (1-based,
//           global row); an exactly zero pivot sets info (first one wins) and
//           skips the scaling, as dgetf2 does.
//   laswp : the panel's row swaps applied to other columns, one thread per
//           column, swaps in pivot order.
//   trsm  : X = L11^-1 X with L11 the panel's unit-lower nb x nb top block,
//           one thread per column of X.
#include <cooperative_groups.h>
#include <stdlib.h>
#include <float.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace lnb {
namespace lu {

constexpr int MAXNB = 32;
constexpr int MAXCL = 8;
constexpr int PT = 512;                 // threads of a panel CTA

// The panel in registers: thread t of CTA q holds rows r0 + t + PT i (i < RPT)
// of the NB-wide panel, a[i][j] its column j.  The column loop is unrolled, so
// every register index is a constant; columns at or past nb are zero and never
// written back.  Per column: warp maxima -> CTA candidate (one barrier) ->
// cluster barrier -> every warp reduces the cluster's candidates -> the owner
// of the pivot row and the owner of row c0+k stage those rows in shared memory
// -> cluster barrier -> every CTA copies the pivot row (the U row) from its
// owner over DSMEM -> barrier -> row k takes the pivot row, the pivot row's
// slot takes the old row k (read from its owner over DSMEM), and every thread
// scales and updates its rows below the pivot.
template <int NB, int RPT>
__global__ void __launch_bounds__(PT) k_lu_panel(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int *piv,
                                                 lnb_status_t *st)
{
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), ncl = (int)cl.num_blocks();
    __shared__ double wv[PT / 32];
    __shared__ long long wi[PT / 32];
    __shared__ double cand[2];              // [0] = |max|, [1] = its global row (-1: none)
    __shared__ double prow[NB], krow[NB];   // pivot row / old row k, at their owners
    __shared__ double urow[NB];             // the pivot row, every CTA
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t r0 = c0 + (int64_t)rank * PT * RPT;
    double a[RPT][NB];
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int64_t g = r0 + tid + (int64_t)PT * i;
#pragma unroll
        for (int j = 0; j < NB; ++j) a[i][j] = (g < m && j < nb) ? A[g + (c0 + j) * lda] : 0.0;
    }

#pragma unroll
    for (int k = 0; k < NB; ++k) {
        if (k >= nb) break;                                   // uniform
        const int64_t gk = c0 + k;
        // 1. candidates: mine, my warp's, my CTA's
        double best = -1.0;
        long long bi = LLONG_MAX;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int64_t g = r0 + tid + (int64_t)PT * i;
            if (g < m && g >= gk) {
                const double v = fabs(a[i][k]);
                if (v > best) { best = v; bi = g; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { wv[warp] = best; wi[warp] = bi; }
        __syncthreads();
        if (warp == 0) {
            best = lane < PT / 32 ? wv[lane] : -1.0;
            bi = lane < PT / 32 ? wi[lane] : LLONG_MAX;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, best, o);
                const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
            }
            if (lane == 0) {
                cand[0] = best;
                cand[1] = bi == LLONG_MAX ? -1.0 : (double)bi;
            }
        }
        if (ncl > 1) cl.sync(); else __syncthreads();          // #1: candidates visible
        // 2. the pivot row, reduced by every warp from the cluster's candidates
        int64_t p;
        {
            double gb = -1.0;
            long long gi = LLONG_MAX;
            if (lane < ncl) {
                const double *cq = cl.map_shared_rank(cand, lane);
                if (cq[1] >= 0.0) { gb = cq[0]; gi = (long long)cq[1]; }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1) {                  // ncl <= 8
                const double ov = __shfl_xor_sync(0xffffffffu, gb, o);
                const long long oi = __shfl_xor_sync(0xffffffffu, gi, o);
                if (ov > gb || (ov == gb && oi < gi)) { gb = ov; gi = oi; }
            }
            p = __shfl_sync(0xffffffffu, gi, 0);
        }
        // 3. the owners stage the two rows
        const int64_t dk = gk - r0, dp = p - r0;               // positions in my slice
        const bool own_k = dk >= 0 && dk < (int64_t)PT * RPT && (int)(dk % PT) == tid;
        const bool own_p = dp >= 0 && dp < (int64_t)PT * RPT && (int)(dp % PT) == tid;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            if (own_p && dp / PT == i)
#pragma unroll
                for (int j = 0; j < NB; ++j) prow[j] = a[i][j];
            if (own_k && dk / PT == i)
#pragma unroll
                for (int j = 0; j < NB; ++j) krow[j] = a[i][j];
        }
        if (ncl > 1) cl.sync(); else __syncthreads();          // #2: both rows staged
        const int ok = (int)((gk - c0) / ((int64_t)PT * RPT)), op = (int)((p - c0) / ((int64_t)PT * RPT));
        if (tid < NB) urow[tid] = *cl.map_shared_rank(prow + tid, op);
        __syncthreads();
        // 4. row k := pivot row, row p := old row k; scale and update the rows below
        const double pv = urow[k];
        if (pv == 0.0 && rank == 0 && tid == 0) atomicCAS(&st->info, 0, (int)(gk + 1));
        const double *kr = cl.map_shared_rank(krow, ok);
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int64_t g = r0 + tid + (int64_t)PT * i;
            if (g == gk) {
#pragma unroll
                for (int j = 0; j < NB; ++j) a[i][j] = urow[j];
            } else if (g == p) {
#pragma unroll
                for (int j = 0; j < NB; ++j) a[i][j] = kr[j];
            }
            if (g < m && g > gk) {
                double l = a[i][k];
                if (pv != 0.0) {
                    l = l / pv;
                    a[i][k] = l;
                }
#pragma unroll
                for (int j = k + 1; j < NB; ++j) a[i][j] -= l * urow[j];
            }
        }
        if (rank == 0 && tid == 0) piv[gk] = (int)(p + 1);
    }
#pragma unroll
    for (int i = 0; i < RPT; ++i) {
        const int64_t g = r0 + tid + (int64_t)PT * i;
        if (g < m)
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) A[g + (c0 + j) * lda] = a[i][j];
    }
    if (ncl > 1) cl.sync();                                  // no CTA leaves while its smem may be read
}

// rows k and piv[k]-1 swap, k = k0..k1-1 in order, on columns [a0, a1) and
// [b0, b1).  Swapping in place would chain every swap's load after the last
// one's store; instead each chunk of up to 32 swaps is first composed into a
// permutation of the (at most 64) rows it touches -- rows[e] receives the old
// contents of row src[e] -- by warp 0 (lane l keeps entries l and l + 32; a
// ballot finds a pivot row among them), then every column thread gathers all
// sources and scatters them: two memory rounds per chunk.
constexpr int SW = 32, SWT = 64;    // 64 threads: the gather buffer is 32 KB of static shared memory
__global__ void __launch_bounds__(SWT) k_laswp(double *A, int64_t lda, int64_t k0, int64_t k1, const int *piv,
                                               int64_t a0, int64_t a1, int64_t b0, int64_t b1)
{
    __shared__ long long rows[2 * SW], src[2 * SW];
    __shared__ int s_cnt;
    __shared__ double vals[2 * SW][SWT];
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * SWT + threadIdx.x;
    const int64_t na = a1 > a0 ? a1 - a0 : 0, nbb = b1 > b0 ? b1 - b0 : 0;
    const bool act = t < na + nbb;
    double *col = act ? A + (t < na ? a0 + t : b0 + (t - na)) * lda : A;
    for (int64_t c0 = k0; c0 < k1; c0 += SW) {
        const int nk = (int)(k1 - c0 < SW ? k1 - c0 : SW);
        if (threadIdx.x < 32) {
            const long long pk = lane < nk ? (long long)__ldg(piv + c0 + lane) - 1 : 0;
            // entry e = lane (chunk row c0 + lane) and e = lane + 32 (an extra row)
            long long rlo = c0 + lane, slo = c0 + lane, rhi = -1, shi = -1;
            int cnt = nk;
            for (int i = 0; i < nk; ++i) {
                const long long p = __shfl_sync(0xffffffffu, pk, i);
                int ip;
                if (p < c0 + nk) {
                    ip = (int)(p - c0);
                } else {
                    const unsigned hit = __ballot_sync(0xffffffffu, rhi == p);
                    if (hit) {
                        ip = 32 + __ffs(hit) - 1;
                    } else {
                        ip = 32 + (cnt - nk);
                        if (lane == ip - 32) { rhi = p; shi = p; }
                        ++cnt;
                    }
                }
                // swap src[i] and src[ip]
                const long long si = __shfl_sync(0xffffffffu, slo, i);
                const long long sp = ip < 32 ? __shfl_sync(0xffffffffu, slo, ip & 31)
                                             : __shfl_sync(0xffffffffu, shi, ip & 31);
                if (lane == i) slo = sp;
                if (ip < 32) { if (lane == ip) slo = si; }
                else if (lane == ip - 32) shi = si;
            }
            // pack: entries 0..nk-1, then the extras
            if (lane < nk) { rows[lane] = rlo; src[lane] = slo; }
            if (lane < cnt - nk) { rows[nk + lane] = rhi; src[nk + lane] = shi; }
            if (lane == 0) s_cnt = cnt;
        }
        __syncthreads();
        const int cnt = s_cnt;
        if (act) {
#pragma unroll 8
            for (int i = 0; i < cnt; ++i) vals[i][threadIdx.x] = col[src[i]];
#pragma unroll 8
            for (int i = 0; i < cnt; ++i) col[rows[i]] = vals[i][threadIdx.x];
        }
        __syncthreads();
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

// Panel width for `rows` rows: NB x RPT = 32 doubles per thread, 512 threads
// per CTA, at most 8 CTAs per cluster: 32 columns up to 4096 rows, 16 up to
// 8192, 8 up to 16384, 4 up to 32768; 0 beyond.
extern "C" int lnb_lu_panel_width(int64_t rows)
{
    for (int nb = MAXNB, rpt = 1; nb >= 4; nb >>= 1, rpt <<= 1)
        if (rows <= (int64_t)MAXCL * PT * rpt) return nb;
    return 0;
}

template <int NB, int RPT>
static int launch_panel(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int *piv, lnb_status_t *st,
                        lnb_stream_t s)
{
    const int64_t rows = m - c0;
    const int ncl = (int)((rows + (int64_t)PT * RPT - 1) / ((int64_t)PT * RPT));
    if (ncl < 1 || ncl > MAXCL || nb > NB) return (int)cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ncl);
    cfg.blockDim = dim3(PT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = (cudaStream_t)s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)ncl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, k_lu_panel<NB, RPT>, A, lda, m, c0, nb, piv, st);
}

extern "C" int lnb_k_lu_panel_f64(double *A, int64_t lda, int64_t m, int64_t c0, int nb, int *piv, lnb_status_t *st,
                                  lnb_stream_t s)
{
    const int64_t rows = m - c0;
    if (rows <= 0 || nb <= 0) return 0;
    const int w = lnb_lu_panel_width(rows);
    if (w == 0 || nb > w) return (int)cudaErrorInvalidValue;
    int e;
    switch (w) {
    case 32: e = launch_panel<32, 1>(A, lda, m, c0, nb, piv, st, s); break;
    case 16: e = launch_panel<16, 2>(A, lda, m, c0, nb, piv, st, s); break;
    case 8: e = launch_panel<8, 4>(A, lda, m, c0, nb, piv, st, s); break;
    default: e = launch_panel<4, 8>(A, lda, m, c0, nb, piv, st, s); break;
    }
    lnb_prof_count(1);
    return e;
}

extern "C" int lnb_k_laswp_f64(double *A, int64_t lda, int64_t k0, int64_t k1, const int *piv, int64_t a0,
                               int64_t a1, int64_t b0, int64_t b1, lnb_stream_t s)
{
    const int64_t ncols = (a1 > a0 ? a1 - a0 : 0) + (b1 > b0 ? b1 - b0 : 0);
    if (ncols <= 0 || k1 <= k0) return 0;
    k_laswp<<<(unsigned)((ncols + SWT - 1) / SWT), SWT, 0, (cudaStream_t)s>>>(A, lda, k0, k1, piv, a0, a1, b0, b1);
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
