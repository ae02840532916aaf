// k_batched.cu -- many independent uneven SPD systems in one persistent launch.
//
// Each system is the reference's SPD solve (dspdsolv_main, spdsolv_main.c:10-20:
// tile Cholesky then the forward and backward solves) followed, in the
// low-precision mode, by the refinement of itref.c (FP64 residual and
// update).  A CTA takes systems from an atomic ticket over a cost-sorted
// order (largest first), so the uneven sizes balance over the SMs; the whole
// batch is one launch and can be captured in a CUDA graph.
//
// Per system (n <= 512, nrhs <= 8), in one CTA of NT threads:
//   1. the lower triangle of A (FP64) goes to the CTA's scratch factor F
//      (type TF = float or double, 16-byte-aligned columns, L2-resident); the
//      same pass forms ||A||_inf from the column sums of the lower part
//   2. right-looking Cholesky in 32-column panels: the panel is staged in
//      shared memory by cp.async, one warp factors its diagonal block
//      left-looking and inverts it, the rows below become dot products with
//      that inverse, and the trailing update runs 4 x 4 tiles per thread with
//      16-byte loads, the C tile fetched before the products so its latency
//      is hidden
//   3. x = 0, r = b; repeat: z = F^-T F^-1 r (32-row blocks: coalesced partial
//      sums over all warps, then the stored block inverse), x += z,
//      r = b - A x in FP64 from the original A (rows x column groups, several
//      loads in flight per thread); stop at backward error
//      ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol, at most max_iter
//      times (one direct solve when TF = double)
#include "k_bfactor.cuh"

namespace lnb {

struct BatchArgs {
    int count;
    const int *n, *nrhs;
    const int64_t *a_off, *b_off;
    const double *A, *B;
    double *X;
    void *scratch;            // per CTA: factor F (BMAXN x BMAXN) then BMAXN/32 inverse blocks (32 x 32)
    const int *order;         // processing order (cost-sorted)
    int *ticket;
    int *info, *iters;
    int max_iter;
    double tol_eps;           // tol = tol_eps * n
};

template <typename TF>
__host__ __device__ constexpr int64_t bscratch_elems() { return (int64_t)BMAXN * BMAXN + (int64_t)(BMAXN / BP) * BP * BP; }

// shared-memory layout of one CTA (bytes).  The panel buffer is dead once the
// factorization is done, so the solve phase keeps r / z and the reduction
// buffer in it: 103 KB for 256 threads in FP32 mode, two systems per SM.
template <typename TF, int NT>
struct BSmem {
    static constexpr size_t P = sizeof(TF) * BP * BLDP;              // panel, P[c][r] (factor phase)
    static constexpr size_t RS = sizeof(double) * BMAXR * BMAXN;      // r, z (solve phase, inside the panel)
    static constexpr size_t RED = sizeof(double) * (NT / 32) * BP * BMAXR;
    static constexpr size_t SD = (size_t)bsd_bytes<TF>();               // staged block inverse (solve phase)
    static constexpr size_t PR = P > RS + RED + SD ? P : RS + RED + SD;
    static constexpr size_t LI = sizeof(TF) * BP * (BP + 1);         // block inverse, Li[p][j] = inv[j][p]
    static constexpr size_t RD = sizeof(TF) * BP;                     // 1 / diagonal
    static constexpr size_t CS = sizeof(float) * BMAXN;               // column sums of |A|
    static constexpr size_t XS = sizeof(double) * BMAXR * BMAXN;      // x
    static constexpr size_t total = PR + LI + RD + CS + XS;
};
// every shape fits one CTA's 227 KB; the autotuner's "two FP32 systems per SM"
// needs two 256-thread CTAs (plus 1 KB reserved each) within the SM's 228 KB
static_assert(BSmem<double, 256>::total <= 227 * 1024 && BSmem<float, 512>::total <= 227 * 1024,
              "batched solver: shared memory per CTA");
static_assert(2 * (BSmem<float, 256>::total + 1024) <= 228 * 1024, "batched solver: two FP32 systems per SM");

// r = b - A x (A full symmetric n x n, FP64) for nr columns; returns the max
// over columns of ||r||_inf / (anorm ||x||_inf + ||b||_inf), same in every thread
template <int NT>
__device__ double bresidual(const double *A, int n, int nr, const double *B, const double *x, double *r,
                            double anorm, double *red)
{
    const int tid = threadIdx.x;
    constexpr int CG = NT / 64;            // column groups
    const int i0 = tid & 63, cg = tid >> 6;
    for (int rb = 0; rb < n; rb += 64) {
        const int i = rb + i0;
        double acc[BMAXR];
#pragma unroll
        for (int q = 0; q < BMAXR; ++q) acc[q] = 0.0;
        if (i < n) {
#pragma unroll 16
            for (int c = cg; c < n; c += CG) {
                const double a = __ldg(A + i + (int64_t)c * n);
#pragma unroll
                for (int q = 0; q < BMAXR; ++q)
                    if (q < nr) acc[q] = fma(a, x[q * BMAXN + c], acc[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < BMAXR; ++q) red[(q * CG + cg) * 64 + i0] = acc[q];   // lanes contiguous
        __syncthreads();
        for (int t = tid; t < 64 * nr; t += NT) {
            const int q = t >> 6, ii = t & 63;
            if (rb + ii < n) {
                double s = 0.0;
                for (int g = 0; g < CG; ++g) s += red[(q * CG + g) * 64 + ii];
                r[q * BMAXN + rb + ii] = B[(rb + ii) + (int64_t)q * n] - s;
            }
        }
        __syncthreads();
    }
    double worst = 0.0;
    for (int q = 0; q < nr; ++q) {
        double rm = 0.0, xm = 0.0, bm = 0.0;
        for (int i = tid; i < n; i += NT) {
            rm = fmax(rm, fabs(r[q * BMAXN + i]));
            xm = fmax(xm, fabs(x[q * BMAXN + i]));
            bm = fmax(bm, fabs(B[i + (int64_t)q * n]));
        }
        rm = bmax_block<NT>(rm, red);
        xm = bmax_block<NT>(xm, red);
        bm = bmax_block<NT>(bm, red);
        const double den = anorm * xm + bm;
        worst = fmax(worst, den > 0.0 ? rm / den : 0.0);
    }
    return worst;
}

template <typename TF, int NT>
__global__ void __launch_bounds__(NT) k_batched_posv(BatchArgs a)
{
    using SM = BSmem<TF, NT>;
    extern __shared__ __align__(16) unsigned char smb[];
    TF *P = (TF *)smb;
    double *rs = (double *)smb;                                   // aliases P: solve phase only
    double *red = (double *)(smb + SM::RS);                       // aliases P: solve phase only
    TF *sD = (TF *)(smb + SM::RS + SM::RED);                      // aliases P: solve phase only
    TF *Li = (TF *)(smb + SM::PR);
    TF *Rd = (TF *)(smb + SM::PR + SM::LI);
    float *colsum = (float *)(smb + SM::PR + SM::LI + SM::RD);
    double *xs = (double *)(smb + SM::PR + SM::LI + SM::RD + SM::CS);
    __shared__ int s_item, s_fail;
    TF *F = (TF *)a.scratch + (int64_t)blockIdx.x * bscratch_elems<TF>();
    TF *Dv = F + (int64_t)BMAXN * BMAXN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
        const int ldF = (n + 3) & ~3;
        // F = lower(A) in TF, and the column sums of |A| (= row sums) from the lower part
        for (int i = tid; i < n; i += NT) colsum[i] = 0.f;
        __syncthreads();
        for (int c = warp; c < n; c += NT / 32) {
            float sc = 0.f;
#pragma unroll 4
            for (int r = c + lane; r < n; r += 32) {
                const double v = __ldg(A + r + (int64_t)c * n);
                F[r + (int64_t)c * ldF] = (TF)v;
                const float av = (float)fabs(v);
                sc += av;
                if (r > c) atomicAdd(&colsum[r], av);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sc += __shfl_down_sync(0xffffffffu, sc, o);
            if (lane == 0) atomicAdd(&colsum[c], sc);
        }
        __syncthreads();
        const int info = bfactor<TF, NT>(F, ldF, n, Dv, P, Li, Rd, &s_fail);
        __syncthreads();                                          // P is free: r / z and red take it over
        int it = 0;
        if (info == 0) {
            double am = 0.0;
            for (int i = tid; i < n; i += NT) am = fmax(am, (double)colsum[i]);
            const double anorm = bmax_block<NT>(am, red);
            for (int t = tid; t < BMAXR * BMAXN; t += NT) xs[t] = 0.0;
            for (int t = tid; t < n * nr; t += NT) {
                const int i = t % n, q = t / n;
                rs[q * BMAXN + i] = B[i + (int64_t)q * n];
            }
            __syncthreads();
            const double tol = a.tol_eps * n;
            const int maxit = (sizeof(TF) == 8) ? 1 : a.max_iter;
            for (it = 1; it <= maxit; ++it) {
                bsolve<TF, NT>(F, ldF, Dv, n, nr, rs, red, sD);       // r <- M^-1 r
                for (int t = tid; t < n * nr; t += NT) {
                    const int i = t % n, q = t / n;
                    xs[q * BMAXN + i] += rs[q * BMAXN + i];
                }
                __syncthreads();
                if (it == maxit && sizeof(TF) == 8) break;             // FP64 factor: one direct solve
                const double worst = bresidual<NT>(A, n, nr, B, xs, rs, anorm, red);
                if (worst <= tol) break;
            }
            if (it > maxit) it = maxit;
            for (int t = tid; t < n * nr; t += NT) {
                const int i = t % n, q = t / n;
                Xo[i + (int64_t)q * n] = xs[q * BMAXN + i];
            }
        }
        if (tid == 0) {
            if (a.info) a.info[sys] = info;
            if (a.iters) a.iters[sys] = it;
        }
        __syncthreads();
    }
}

// processing order: systems by decreasing n (a counting sort; one CTA).
// interleave: the k-th largest goes to position 2k for the larger half and
// the rest fill the odd positions smallest first (largest, smallest, second
// largest, ...), so CTAs sharing an SM mix long and short systems.
__global__ void __launch_bounds__(1024) k_batch_order(int count, const int *n, int *order, int interleave)
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
        const int k = atomicAdd(&hist[v], 1);
        const int pos = !interleave ? k : (k < (count + 1) / 2 ? 2 * k : 2 * (count - 1 - k) + 1);
        order[pos] = s;
    }
}

}  // namespace lnb

using namespace lnb;

extern "C" int lnb_k_batch_order(int count, const int *n, int *order, int interleave, lnb_stream_t s)
{
    k_batch_order<<<1, 1024, 0, s>>>(count, n, order, interleave);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

extern "C" size_t lnb_batched_scratch_bytes(int grid, int fp64)
{
    return (size_t)grid * (fp64 ? bscratch_elems<double>() * 8 : bscratch_elems<float>() * 4);
}

template <typename TF, int NT>
static void launch_batched(const BatchArgs &a, int grid, lnb_stream_t s)
{
    const int smem = (int)BSmem<TF, NT>::total;
    cudaFuncSetAttribute(k_batched_posv<TF, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_batched_posv<TF, NT><<<grid, NT, smem, s>>>(a);
}

// variant: CTA size, 256 or 512 threads (512 in FP32 mode only)
extern "C" int lnb_k_batched_posv(int count, const int *n, const int *nrhs, const int64_t *a_off,
                                  const int64_t *b_off, const double *A, const double *B, double *X, void *scratch,
                                  int grid, const int *order, int *ticket, int *info, int *iters, int max_iter,
                                  int fp64, int variant, lnb_stream_t s)
{
    BatchArgs a;
    a.count = count; a.n = n; a.nrhs = nrhs; a.a_off = a_off; a.b_off = b_off; a.A = A; a.B = B; a.X = X;
    a.scratch = scratch; a.order = order; a.ticket = ticket; a.info = info; a.iters = iters;
    /* refinement stops at 5 n u: half the reported bar of 10 n u, so that an
     * independent FP64 residual (another summation order) stays under it */
    a.max_iter = max_iter; a.tol_eps = 5.0 * 1.1102230246251565e-16;
    if ((uintptr_t)scratch % 16) return (int)cudaErrorMisalignedAddress;
    cudaError_t e = cudaMemsetAsync(ticket, 0, sizeof(int), s);
    if (e != cudaSuccess) return (int)e;
    if (fp64) launch_batched<double, 256>(a, grid, s);
    else if (variant == 512) launch_batched<float, 512>(a, grid, s);
    else launch_batched<float, 256>(a, grid, s);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
