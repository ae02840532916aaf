// k_sparse.cu -- kernels of the sparse refinement (itref.c built with
// USE_SPARSE): the CSR product and the block-Jacobi preconditioner.
//
//   csrmv   : y = alpha A x + beta y over a CSR matrix (zero- or one-based);
//             8 lanes per row, each row's products summed in a fixed order
//             (lane-strided partial sums, then a fixed shuffle tree), so the
//             result does not depend on scheduling.  The reference's
//             bsblas_dcsrmv (bsblas_csrmm.h:214-232) is MKL's mkl_dcsrmv.
//   bj_*    : the preconditioner of itref_setup.c:55-93: the complete
//             diagonal blocks of order bm (hb_sym_diag_block, hb.c:512) made
//             dense, each factored by Cholesky with natural ordering (what
//             cs_schol(A, 0) + cs_chol compute) by one CTA with the batched
//             solver's bfactor, and applied as z = L^-T L^-1 r
//             (bsblas_dcholsolv2, bsblas_csrmm.h:498) with its bsolve.
#include <climits>

#include "k_bfactor.cuh"

namespace lnb {
namespace sp {

constexpr int RL = 8;            // lanes per row of the CSR product
constexpr int NT = 256;

__global__ void __launch_bounds__(NT) k_csrmv(int64_t n, int base, const int *__restrict__ vptr,
                                              const int *__restrict__ vpos, const double *__restrict__ vval,
                                              const double *__restrict__ x, double alpha, double beta,
                                              const double *yin, double *y)
{
    const int lane = threadIdx.x & (RL - 1);
    const int64_t rows_per_grid = (int64_t)gridDim.x * (NT / RL);
    for (int64_t i = (int64_t)blockIdx.x * (NT / RL) + threadIdx.x / RL; i < n; i += rows_per_grid) {
        const int p0 = vptr[i] - base, p1 = vptr[i + 1] - base;
        double s = 0.0;
        for (int p = p0 + lane; p < p1; p += RL) s = fma(vval[p], __ldg(x + (vpos[p] - base)), s);
#pragma unroll
        for (int o = RL / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, RL);
        if (lane == 0) y[i] = (beta == 0.0 ? 0.0 : beta * yin[i]) + alpha * s;
    }
}

// per-block layout of the factors: F (bk x bk, ld ldF) then the 32 x 32
// inverses of its diagonal blocks
__host__ __device__ inline int64_t bj_ldf(int bm) { return ((int64_t)bm + 3) & ~(int64_t)3; }
__host__ __device__ inline int64_t bj_stride(int bm)
{
    return bj_ldf(bm) * bm + (int64_t)((bm + BP - 1) / BP) * BP * BP;
}

// the envelope of block k's factor, per 32-row tile (bsolve's env): with natural
// ordering the Cholesky factor keeps every row's nonzeros at or right of the
// row's first nonzero in A (L_ij = (0 - sum of zeros) / L_jj = 0 before it)
constexpr int ENV = 2 * (lnb::BMAXN / lnb::BP);

// block k of the matrix, dense: F[(r - r0) + (c - r0) ldF] for r, c in [r0, r0 + bk);
// env[k * ENV ..] its factor's envelope
__global__ void __launch_bounds__(NT) k_bj_densify(int64_t n, int bm, int base, const int *__restrict__ vptr,
                                                   const int *__restrict__ vpos, const double *__restrict__ vval,
                                                   double *fac, int *env)
{
    constexpr int NTL = lnb::BMAXN / lnb::BP;
    __shared__ int first[NTL], last[NTL];
    if (threadIdx.x < NTL) { first[threadIdx.x] = INT_MAX; last[threadIdx.x] = -1; }
    const int64_t k = blockIdx.x, r0 = k * bm;
    const int bk = (int)((n - r0) < bm ? (n - r0) : bm);
    const int64_t ldF = bj_ldf(bm);
    double *F = fac + k * bj_stride(bm);
    for (int64_t i = threadIdx.x; i < ldF * bk; i += NT) F[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < bk; r += NT / 32) {
        const int p0 = vptr[r0 + r] - base, p1 = vptr[r0 + r + 1] - base;
        int f = r;                                          // the diagonal at least
        for (int p = p0 + lane; p < p1; p += 32) {
            const int64_t c = (int64_t)vpos[p] - base;
            if (c >= r0 && c < r0 + bk) {
                atomicAdd(F + r + (c - r0) * ldF, vval[p]);
                if (c - r0 < f) f = (int)(c - r0);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) f = min(f, __shfl_xor_sync(0xffffffffu, f, o));
        if (lane == 0) {
            atomicMin(&first[r / lnb::BP], f);
            for (int t = f / lnb::BP; t <= r / lnb::BP; ++t) atomicMax(&last[t], r);
        }
    }
    __syncthreads();
    if (threadIdx.x < NTL) {
        env[k * ENV + threadIdx.x] = first[threadIdx.x] == INT_MAX ? 0 : first[threadIdx.x];
        env[k * ENV + NTL + threadIdx.x] = last[threadIdx.x];
    }
}

struct BjSmem {
    static constexpr size_t P = sizeof(double) * BP * BLDP;
    static constexpr size_t LI = sizeof(double) * BP * (BP + 1);
    static constexpr size_t RD = sizeof(double) * BP;
    static constexpr size_t total = P + LI + RD;
};

// factor every block (one CTA each); info[k] = 0 or the 1-based failing pivot
__global__ void __launch_bounds__(NT) k_bj_factor(int64_t n, int bm, double *fac, int *info)
{
    extern __shared__ __align__(16) unsigned char smb[];
    double *P = (double *)smb;
    double *Li = (double *)(smb + BjSmem::P);
    double *Rd = (double *)(smb + BjSmem::P + BjSmem::LI);
    __shared__ int s_fail;
    const int64_t k = blockIdx.x, r0 = k * bm;
    const int bk = (int)((n - r0) < bm ? (n - r0) : bm);
    const int64_t ldF = bj_ldf(bm);
    double *F = fac + k * bj_stride(bm);
    double *Dv = F + ldF * bm;
    const int f = bfactor<double, NT>(F, (int)ldF, bk, Dv, P, Li, Rd, &s_fail);
    if (threadIdx.x == 0) info[k] = f;
}

// z = M^-1 r, one CTA per block
__global__ void __launch_bounds__(NT) k_bj_apply(int64_t n, int bm, const double *fac, const int *env,
                                                 const double *r, double *z)
{
    __shared__ double zs[BMAXN];
    __shared__ double red[(NT / 32) * BP * BMAXR];
    __shared__ __align__(16) double sD[bsd_bytes<double>() / sizeof(double)];
    const int64_t k = blockIdx.x, r0 = k * bm;
    const int bk = (int)((n - r0) < bm ? (n - r0) : bm);
    const int64_t ldF = bj_ldf(bm);
    const double *F = fac + k * bj_stride(bm);
    for (int i = threadIdx.x; i < bk; i += NT) zs[i] = r[r0 + i];
    __syncthreads();
    bsolve<double, NT>(F, (int)ldF, F + ldF * bm, bk, 1, zs, red, sD, env + k * ENV);
    for (int i = threadIdx.x; i < bk; i += NT) z[r0 + i] = zs[i];
}

}  // namespace sp
}  // namespace lnb

extern "C" int lnb_k_csrmv_f64(int64_t n, int base, const int *vptr, const int *vpos, const double *vval,
                               const double *x, double alpha, double beta, const double *yin, double *y,
                               lnb_stream_t s)
{
    using namespace lnb::sp;
    if (n <= 0) return 0;
    const int64_t blocks = (n + NT / RL - 1) / (NT / RL);
    k_csrmv<<<(unsigned)(blocks < 8192 ? blocks : 8192), NT, 0, (cudaStream_t)s>>>(n, base, vptr, vpos, vval, x, alpha,
                                                                                 beta, yin, y);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" int64_t lnb_bj_doubles(int64_t n, int bm)
{
    return ((n + bm - 1) / bm) * lnb::sp::bj_stride(bm);
}
extern "C" int64_t lnb_bj_env_ints(int64_t n, int bm) { return ((n + bm - 1) / bm) * lnb::sp::ENV; }

// densify and factor the diagonal blocks; info[nblk] receives each block's info
extern "C" int lnb_k_bj_setup(int64_t n, int bm, int base, const int *vptr, const int *vpos, const double *vval,
                              double *fac, int *env, int *info, lnb_stream_t s)
{
    using namespace lnb::sp;
    if (n <= 0) return 0;
    if (bm < 1 || bm > lnb::BMAXN) return (int)cudaErrorInvalidValue;
    const unsigned nblk = (unsigned)((n + bm - 1) / bm);
    k_bj_densify<<<nblk, NT, 0, (cudaStream_t)s>>>(n, bm, base, vptr, vpos, vval, fac, env);
    cudaError_t e = cudaFuncSetAttribute(k_bj_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BjSmem::total);
    if (e != cudaSuccess) return (int)e;
    k_bj_factor<<<nblk, NT, BjSmem::total, (cudaStream_t)s>>>(n, bm, fac, info);
    lnb_prof_count(2);
    return (int)cudaGetLastError();
}

extern "C" int lnb_k_bj_apply(int64_t n, int bm, const double *fac, const int *env, const double *r, double *z,
                              lnb_stream_t s)
{
    using namespace lnb::sp;
    if (n <= 0) return 0;
    k_bj_apply<<<(unsigned)((n + bm - 1) / bm), NT, 0, (cudaStream_t)s>>>(n, bm, fac, env, r, z);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
