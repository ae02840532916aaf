// k_trsv_blk.cu -- triangular solves with an FP32 lower factor and few
// right-hand sides (1..8), FP64 vectors and arithmetic, built on the inverses
// of the factor's HB x HB diagonal blocks (HB = 512).
//
// Semantics of the two blocked solves of dspdsolv_main (spdsolv_main.c:15,17,
// bblas_dltrsm bblas_trsm.h:119-160): forward L y = b walks block rows top
// down, y_s = L_ss^-1 (b_s - sum_{j<s} L_sj y_j); backward L^T x = y walks them
// bottom up, x_s = L_ss^-T (y_s - sum_{j>s} L_js^T x_j).  With the diagonal
// blocks inverted beforehand every step is matrix-vector work:
//
//   * Work items are 64 KB slabs: 64 rows x 256 columns (forward) or 256 rows
//     x 64 columns (backward) of an HB x HB block (16 items per block), each
//     brought into shared memory by 2 (forward) or 8 (backward) 2D TMA boxes
//     of 128-byte swizzled rows on one mbarrier, issued before the item waits
//     for its input vector.  An item multiplies its slab by a segment of up to
//     8 vectors on the FP64 tensor cores (DMMA, FP32 widened as it loads) and
//     adds the product into a target segment with FP64 atomics, then bumps a
//     counter: the residual counter of the target block row (update items,
//     L_sj y_j or L_js^T x_j) or the solution counter of the step (diagonal
//     items, with L_ss^-1 or L_ss^-T).
//   * Items are handed out by an atomic ticket in a topological order that
//     puts the chain first: step k holds the diagonal items of block s, the
//     items that feed the next block row, then the bulk of the column one
//     step behind (its remaining rows).  Every item waits only on items of
//     earlier steps or earlier in its own step, which running CTAs hold, so the
//     walk cannot deadlock whatever the residency.  All waits are bounded and
//     report a site code; a CTA that gives up drains its TMA load first.
//   * The chain is nb = n/HB steps long (64 at n = 32768), against n/64 for a
//     substitution with 64-wide blocks, and the bulk streams the factor once.
//
// The block inverses come from lnb_k_trtri_hb_f32 (this file): FP64
// arithmetic, FP32 storage, built column block by column block from the
// 64 x 64 inverses of lnb_k_trtri_blocks_f32.
#include <stdlib.h>
#include <string.h>

#include "common.cuh"
#include "tc_sm100.cuh"

namespace lnb {
namespace blk {

constexpr int NTHR = 256;
constexpr int SLAB = 64 * 256;        // floats per item slab (64 KB)
constexpr int MAXR = 8;               // right-hand sides per launch

struct Args {
    int64_t n, np;          // order, padded order nb * HB
    int nb, nrhs, fwd, nitems;
    int hb, ipb;            // diagonal block order HB, items per block (HB / 64) (HB / 256)
    double *R, *Y;          // np x nrhs each (ld np): residual right-hand side, solution
    int *ticket, *cntR, *cntY;
    lnb_status_t *st;
    long long wait_ns;
};

// items of step k: ipb diagonal, ipb next-row (k < nb-1), ipb per bulk row (k >= 1: nb-1-k rows)
__host__ __device__ inline int64_t step_start(int64_t k, int64_t nb, int64_t ipb)
{
    const int64_t m = k < nb - 1 ? k : nb - 1;
    const int64_t bulk = k >= 1 ? (k - 1) * (nb - 1) - (k - 1) * k / 2 : 0;
    return ipb * (k + m + bulk);
}

struct Item {
    int kind;     // 0 diagonal, 1 update
    int row;      // target block row (residual for updates, solution for diagonal)
    int col;      // source block column (its solution segment is the input of an update)
    int part;     // 0 .. ipb-1
};

LNB_DEV Item decode(int64_t t, const Args &a)
{
    int lo = 0, hi = a.nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (step_start(mid, a.nb, a.ipb) <= t) lo = mid; else hi = mid - 1;
    }
    const int k = lo;
    int64_t r = t - step_start(k, a.nb, a.ipb);
    const int s = a.fwd ? k : a.nb - 1 - k;           // block solved at this step
    Item it;
    it.part = (int)(r % a.ipb);
    if (r < a.ipb) { it.kind = 0; it.row = s; it.col = s; return it; }
    r -= a.ipb;
    it.kind = 1;
    if (k < a.nb - 1) {
        if (r < a.ipb) {                              // the next block row's last update
            it.row = a.fwd ? s + 1 : s - 1;
            it.col = s;
            return it;
        }
        r -= a.ipb;
    }
    const int off = (int)(r / a.ipb);                 // bulk of the column one step behind
    it.row = a.fwd ? s + 1 + off : s - 1 - off;
    it.col = a.fwd ? s - 1 : s + 1;
    return it;
}

// bounded wait for this CTA's own TMA load; used on the way out after a give-up
LNB_DEV void drain(uint64_t *bar, uint32_t parity, long long wait_ns)
{
    const uint64_t t0 = globaltimer();
    while (!tc::mbar_try_wait(bar, parity)) {
        if ((long long)(globaltimer() - t0) > wait_ns) break;
    }
}

// Slab layout.  The slab arrives as boxes of 32 floats along its contiguous
// (inner) index r, written by TMA with the 128-byte swizzle: box r / 32,
// then one 128-byte row per outer index c, 16-byte chunk (r % 32) / 4 stored
// at chunk position ((r % 32) / 4) ^ (c % 8).  OUTER = 256 (forward: r = the
// 64 outputs, c = the 256 inputs) or 64 (backward: r = the 256 inputs, c =
// the 64 outputs).  With the swizzle the backward A fragments are free of
// bank conflicts and the forward ones 2-way.
template <int OUTER>
LNB_DEV int soff(int r, int c)
{
    return (r >> 5) * (32 * OUTER) + c * 32 + ((((r & 31) >> 2) ^ (c & 7)) << 2) + (r & 3);
}
// x segment element (k, q), 8 columns per row, swizzled so that the B
// fragment loads (rows 4kk + t, column g) are free of bank conflicts
LNB_DEV int voff(int k, int q) { return k * 8 + (q ^ (((k >> 1) & 1) << 2)); }

constexpr int RED_DOUBLES = 64 * 8;
constexpr int BLK_SMEM = 1024 + SLAB * 4 + 256 * 8 * 8 + RED_DOUBLES * 8;

// Item product on the FP64 tensor cores: out (64 x 8) = S (64 x 256) v (256 x 8),
// S = the slab (forward) or its transpose (backward), FP32 widened as the
// fragments load.  Warp w takes output rows 16 (w % 4) .. +15 over inputs
// 128 (w / 4) .. +127 (32 DMMAs); the two input halves meet in shared memory.
__global__ void __launch_bounds__(NTHR, 2) k_trsm_blk(Args a, const __grid_constant__ CUtensorMap mT,
                                                      const __grid_constant__ CUtensorMap mI)
{
    extern __shared__ __align__(16) unsigned char smb[];
    // TMA with the 128-byte swizzle writes to 1024-byte aligned boxes
    const uint32_t base = smem_u32(smb);
    float *slab = reinterpret_cast<float *>(smb + (((base + 1023u) & ~1023u) - base));
    double *vs = reinterpret_cast<double *>(slab + SLAB);          // [256][8] input segment (voff)
    double *red = vs + 256 * 8;                                    // [64][8] partial sums
    __shared__ __align__(8) uint64_t full;
    __shared__ int s_t, s_ok;
    __shared__ volatile int s_abort;     // stays 0: nothing else cuts the slab wait short
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
    if (tid == 0) {
        s_abort = 0;
        tc::mbar_init(&full, 1);
        tc::fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (tid == 0) s_t = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int64_t t = s_t;
        if (t >= a.nitems) break;
        const Item it = decode(t, a);
        // source box and the vector / target segments of this item: 64-wide
        // output slab po, 256-wide input slab pi
        //   forward : slab rows = 64 outputs, columns = 256 inputs
        //   backward: slab rows = 256 inputs, columns = 64 outputs
        const int po = it.part % (a.hb / 64), pi = it.part / (a.hb / 64);
        const int64_t in0 = (int64_t)it.col * a.hb + 256 * pi;
        const int64_t out0 = (int64_t)it.row * a.hb + 64 * po;
        if (tid == 0) {
            tc::mbar_arrive_expect_tx(&full, SLAB * 4);
            const CUtensorMap *m = it.kind == 0 ? &mI : &mT;
            // diagonal items read block s of the inverses (rows 0..HB-1 of
            // column block s), updates L_{row, col} (forward) or L_{col, row}
            int x0, y0;
            if (it.kind == 0) {
                x0 = a.fwd ? 64 * po : 256 * pi;
                y0 = it.row * a.hb + (a.fwd ? 256 * pi : 64 * po);
            } else {
                x0 = a.fwd ? (int)out0 : (int)in0;
                y0 = a.fwd ? (int)in0 : (int)out0;
            }
            if (a.fwd) {
                for (int b = 0; b < 2; ++b) tc::tma_load_2d(slab + b * 32 * 256, m, &full, x0 + 32 * b, y0);
            } else {
                for (int b = 0; b < 8; ++b) tc::tma_load_2d(slab + b * 32 * 64, m, &full, x0 + 32 * b, y0);
            }
            // the input: a solution segment (updates) or a finished residual (diagonal)
            bool ok;
            if (it.kind == 1) {
                ok = wait_geq(a.cntY + it.col, a.ipb, a.wait_ns, a.st);
            } else {
                const int need = a.ipb * (a.fwd ? it.row : a.nb - 1 - it.row);
                ok = wait_geq(a.cntR + it.row, need, a.wait_ns, a.st);
            }
            if (!ok && atomicCAS(&a.st->timeout, 0, it.kind == 0 ? 41 : 42) == 0) a.st->timeout_item = (int)t;
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) drain(&full, phase, a.wait_ns);
            break;
        }
        const double *src = it.kind == 1 ? a.Y : a.R;
        for (int i = tid; i < 8 * 256; i += NTHR) {
            const int q = i >> 8, c = i & 255;
            vs[voff(c, q)] = q < a.nrhs ? __ldcg(src + in0 + c + (int64_t)q * a.np) : 0.0;
        }
        if (tid == 0 && !tc::mbar_wait(&full, phase, a.wait_ns, &s_abort, a.st)) {
            if (atomicCAS(&a.st->timeout, 0, 43) == 0) a.st->timeout_item = (int)t;
            s_ok = 0;
        }
        __syncthreads();
        phase ^= 1;
        if (!s_ok) break;
        const int m16 = (warp & 3) * 16, k00 = (warp >> 2) * 128;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        if (a.fwd) {
#pragma unroll 8
            for (int kk = 0; kk < 32; ++kk) {
                const int k = k00 + 4 * kk + t4;
                const double a0 = (double)slab[soff<256>(m16 + g, k)];
                const double a1 = (double)slab[soff<256>(m16 + g + 8, k)];
                dmma16x8x4(acc, a0, a1, vs[voff(k, g)]);
            }
        } else {
#pragma unroll 8
            for (int kk = 0; kk < 32; ++kk) {
                const int k = k00 + 4 * kk + t4;
                const double a0 = (double)slab[soff<64>(k, m16 + g)];
                const double a1 = (double)slab[soff<64>(k, m16 + g + 8)];
                dmma16x8x4(acc, a0, a1, vs[voff(k, g)]);
            }
        }
        // C fragment: rows m16 + g (+8), columns 2 t4 (+1)
        const int ra = m16 + g, rb = ra + 8, q0 = 2 * t4, q1 = q0 + 1;
        if (warp >= 4) {
            red[ra * 8 + q0] = acc[0];
            red[ra * 8 + q1] = acc[1];
            red[rb * 8 + q0] = acc[2];
            red[rb * 8 + q1] = acc[3];
        }
        __syncthreads();
        if (warp < 4) {
            double *dst = (it.kind == 1 ? a.R : a.Y) + out0;
            const double sg = it.kind == 1 ? -1.0 : 1.0;
            if (q0 < a.nrhs) {
                atomicAdd(dst + ra + (int64_t)q0 * a.np, sg * (acc[0] + red[ra * 8 + q0]));
                atomicAdd(dst + rb + (int64_t)q0 * a.np, sg * (acc[2] + red[rb * 8 + q0]));
            }
            if (q1 < a.nrhs) {
                atomicAdd(dst + ra + (int64_t)q1 * a.np, sg * (acc[1] + red[ra * 8 + q1]));
                atomicAdd(dst + rb + (int64_t)q1 * a.np, sg * (acc[3] + red[rb * 8 + q1]));
            }
        }
        // publish: every thread's atomics, then one GPU-scope release of the counter
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(it.kind == 1 ? a.cntR + it.row : a.cntY + it.row, 1);
        }
    }
}

// R = B (rows < n, zero past n), Y = 0, both np x nrhs
__global__ void k_blk_pack(const double *B, int64_t ldb, int64_t n, int64_t np, int nrhs, double *R, double *Y)
{
    const int q = blockIdx.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < np; r += (int64_t)gridDim.x * blockDim.x) {
        R[r + q * np] = r < n ? B[r + q * ldb] : 0.0;
        Y[r + q * np] = 0.0;
    }
}
__global__ void k_blk_unpack(const double *Y, int64_t n, int64_t np, double *B, int64_t ldb)
{
    const int q = blockIdx.y;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
        B[r + q * ldb] = Y[r + q * np];
}

// ---- the HB x HB diagonal-block inverses -------------------------------------
// CTA (cb, s): column block cb (64 wide) of inv(L_ss), s = block index.  With
// X_a the 64 x 64 block (a, cb) of the inverse and D_a the inverse of the 64 x
// 64 diagonal block a:  X_cb = D_cb,  X_a = -D_a sum_{c=cb}^{a-1} L_ac X_c.
// FP64 arithmetic on operands widened once as they are staged, FP32 storage
// (the earlier X_c are read back as stored).  Rows and columns at or past n
// are the identity's.
constexpr int TLD = 68;
constexpr int TRTRI_SMEM = 3 * 64 * TLD * 8;

template <int HB>
__global__ void __launch_bounds__(256) k_trtri_hb(const float *__restrict__ T, int64_t ldt, int64_t n,
                                                  const float *__restrict__ dinv64, float *Binv)
{
    extern __shared__ __align__(16) double tsm[];
    double (*As)[TLD] = reinterpret_cast<double (*)[TLD]>(tsm);                 // As[k][r] = A[r][k]
    double (*Bs)[TLD] = reinterpret_cast<double (*)[TLD]>(tsm + 64 * TLD);      // Bs[k][c] = B[k][c]
    double (*Cs)[TLD] = reinterpret_cast<double (*)[TLD]>(tsm + 128 * TLD);     // the sum, row-major
    const int cb = blockIdx.x, s = blockIdx.y, tid = threadIdx.x;
    const int64_t o = (int64_t)s * HB;           // first row / column of the block
    const int64_t nb64 = (n + 63) / 64;
    float *Xb = Binv + (int64_t)s * HB * HB;     // block s: element (r, c) at Xb[r + c * HB]
    // blocks above the diagonal are zero
    for (int a = 0; a < cb; ++a)
        for (int i = tid; i < 64 * 64; i += 256) {
            const int c = i >> 6, r = i & 63;
            Xb[(64 * a + r) + (int64_t)(64 * cb + c) * HB] = 0.f;
        }
    // DMMA tiling of a 64 x 64 product: warp w owns rows m0 .. m0+15 and
    // columns n0 .. n0+31 (4 fragments of 8); with the row stride TLD = 68 (4
    // mod 16 doubles) the fragment loads of each half-warp hit distinct banks
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
    const int m0 = 16 * (warp & 3), n0 = 32 * (warp >> 2);
    for (int a = cb; a < HB / 64; ++a) {
        const int64_t q64 = (o + 64 * a) / 64;      // global 64-block index of diagonal block a
        if (a == cb) {
            // X_cb = D_cb (the identity past the 64-blocks of the factor)
            for (int i = tid; i < 64 * 64; i += 256) {
                const int c = i >> 6, r = i & 63;
                Xb[(64 * a + r) + (int64_t)(64 * cb + c) * HB] =
                    q64 < nb64 ? dinv64[q64 * 4096 + r + 64 * c] : (r == c ? 1.f : 0.f);
            }
            __syncthreads();
            continue;
        }
        double acc[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[j][v] = 0.0;
        // sum_{c=cb}^{a-1} L_ac X_c
        for (int c = cb; c < a; ++c) {
            __syncthreads();
            for (int i = tid; i < 64 * 64; i += 256) {
                const int k = i >> 6, r = i & 63;
                const int64_t gr = o + 64 * a + r, gc = o + 64 * c + k;
                As[k][r] = (gr < n && gc < n) ? (double)T[gr + gc * ldt] : 0.0;
                const int cc = i >> 6, kk = i & 63;
                Bs[kk][cc] = (double)Xb[(64 * c + kk) + (int64_t)(64 * cb + cc) * HB];
            }
            __syncthreads();
#pragma unroll 4
            for (int k = 0; k < 64; k += 4) {
                const double a0 = As[k + t4][m0 + g], a1 = As[k + t4][m0 + g + 8];
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma16x8x4(acc[j], a0, a1, Bs[k + t4][n0 + 8 * j + g]);
            }
        }
        // X_a = -D_a * acc   (D_a = identity past the 64-blocks of the factor)
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cc = n0 + 8 * j + 2 * t4;
            Cs[m0 + g][cc] = acc[j][0];
            Cs[m0 + g][cc + 1] = acc[j][1];
            Cs[m0 + g + 8][cc] = acc[j][2];
            Cs[m0 + g + 8][cc + 1] = acc[j][3];
        }
        for (int i = tid; i < 64 * 64; i += 256) {
            const int k = i >> 6, r = i & 63;          // As[k][r] = D_a[r][k]
            As[k][r] = q64 < nb64 ? (double)dinv64[q64 * 4096 + r + 64 * k] : (r == k ? 1.0 : 0.0);
        }
        __syncthreads();
        double out[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) out[j][v] = 0.0;
#pragma unroll 4
        for (int k = 0; k < 64; k += 4) {
            const double a0 = As[k + t4][m0 + g], a1 = As[k + t4][m0 + g + 8];
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma16x8x4(out[j], a0, a1, Cs[k + t4][n0 + 8 * j + g]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int cc = n0 + 8 * j + 2 * t4;
            float *x = Xb + 64 * a + m0 + g + (int64_t)(64 * cb + cc) * HB;
            x[0] = (float)(-out[j][0]);
            x[HB] = (float)(-out[j][1]);
            x[8] = (float)(-out[j][2]);
            x[HB + 8] = (float)(-out[j][3]);
        }
        // the stores of X_a are read back as B operands by the next rows
        __syncthreads();
    }
}

typedef CUresult (*EncodeTiledFnB)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// FP32 rows x cols column-major (ld elements) as a 2D tensor map with bx x by
// boxes (bx = 32 floats = 128 bytes), written with the 128-byte swizzle
static int map2d(CUtensorMap *m, const void *base, int64_t rows, int64_t cols, int64_t ld, int bx, int by)
{
    static EncodeTiledFnB fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return -1;
        fn = (EncodeTiledFnB)p;
    }
    cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
    cuuint32_t box[2] = {(cuuint32_t)bx, (cuuint32_t)by};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

static int launch(const Args &a, const CUtensorMap &mT, const CUtensorMap &mI, int sms, cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(k_trsm_blk, cudaFuncAttributeMaxDynamicSharedMemorySize, BLK_SMEM);
    if (e != cudaSuccess) return (int)e;
    const int grid = a.nitems < 2 * sms ? a.nitems : 2 * sms;
    k_trsm_blk<<<grid, NTHR, BLK_SMEM, s>>>(a, mT, mI);
    return (int)cudaGetLastError();
}

}  // namespace blk
}  // namespace lnb

// diagonal block order of the block solve.  512: with 1024 the chain halves
// but the solve was measured only 5 % faster (its bulk streaming, not the
// chain, sets the time) while the inverses cost 4x the time.
static inline int64_t hb_of(int64_t n) { (void)n; return 512; }

extern "C" int64_t lnb_trsm_blk_ints(int64_t n)
{
    const int64_t nb = (n + hb_of(n) - 1) / hb_of(n);
    return 32 + 2 * nb;
}
extern "C" int64_t lnb_trsm_blk_inv_floats(int64_t n)
{
    const int64_t hb = hb_of(n), nb = (n + hb - 1) / hb;
    return nb * hb * hb;
}
extern "C" int64_t lnb_trsm_blk_vec_doubles(int64_t n, int64_t nrhs)
{
    const int64_t hb = hb_of(n), nb = (n + hb - 1) / hb;
    return 2 * nb * hb * nrhs;
}
// the block solve applies: FP32 T 16-byte aligned with ld a multiple of 4, 1..8 right-hand sides
extern "C" int lnb_trsm_blk_ok(const float *T, int64_t ldt, int64_t n, int64_t nrhs)
{
    const char *e = getenv("LNB_TRSM_BLK");    /* 0: substitution with 64-wide blocks instead */
    if (e && *e && atoi(e) == 0) return 0;
    return n >= 1024 && nrhs >= 1 && nrhs <= lnb::blk::MAXR && (uintptr_t)T % 16 == 0 && ldt % 4 == 0;
}

// Binv: lnb_trsm_blk_inv_floats(n); dinv64: lnb_k_trtri_blocks_f32's 64 x 64 inverses of T
extern "C" int lnb_k_trtri_hb_f32(const float *T, int64_t ldt, int64_t n, const float *dinv64, float *Binv,
                                  lnb_stream_t s)
{
    using namespace lnb::blk;
    if (n <= 0) return 0;
    const int64_t hb = hb_of(n), nb = (n + hb - 1) / hb;
    cudaError_t e = cudaFuncSetAttribute(k_trtri_hb<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, TRTRI_SMEM);
    if (e != cudaSuccess) return (int)e;
    k_trtri_hb<512><<<dim3((unsigned)(hb / 64), (unsigned)nb), 256, TRTRI_SMEM, (cudaStream_t)s>>>(T, ldt, n, dinv64,
                                                                                                  Binv);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

// op(T) X = B in place for lower T (trans 'N': forward, 'T': backward), B n x nrhs
// FP64 (ld ldb); vec: lnb_trsm_blk_vec_doubles(n, nrhs) doubles; sync:
// lnb_trsm_blk_ints(n) ints (zeroed here)
extern "C" int lnb_k_trsm_blk_f32(char trans, int64_t n, int64_t nrhs, const float *T, int64_t ldt, const float *Binv,
                                  double *B, int64_t ldb, double *vec, int *sync, lnb_status_t *st, long long wait_ns,
                                  int sms, lnb_stream_t s)
{
    using namespace lnb::blk;
    if (n <= 0 || nrhs <= 0) return 0;
    if (nrhs > MAXR) return (int)cudaErrorInvalidValue;
    Args a;
    a.n = n;
    a.hb = (int)hb_of(n);
    a.ipb = (a.hb / 64) * (a.hb / 256);
    a.nb = (int)((n + a.hb - 1) / a.hb);
    a.np = (int64_t)a.nb * a.hb;
    a.nrhs = (int)nrhs;
    a.fwd = trans == 'N';
    a.nitems = (int)step_start(a.nb, a.nb, a.ipb);
    a.R = vec;
    a.Y = vec + a.np * nrhs;
    a.ticket = sync;
    a.cntR = sync + 32;
    a.cntY = sync + 32 + a.nb;
    a.st = st;
    a.wait_ns = wait_ns;
    CUtensorMap mT, mI;
    memset(&mT, 0, sizeof mT);
    memset(&mI, 0, sizeof mI);
    // forward items read 2 boxes of 32 x 256, backward 8 boxes of 32 x 64
    const int bx = 32, by = a.fwd ? 256 : 64;
    if (map2d(&mT, T, n, n, ldt, bx, by) || map2d(&mI, Binv, a.hb, a.np, a.hb, bx, by))
        return (int)cudaErrorInvalidValue;
    cudaStream_t cs = (cudaStream_t)s;
    cudaError_t e = cudaMemsetAsync(sync, 0, (size_t)lnb_trsm_blk_ints(n) * sizeof(int), cs);
    if (e != cudaSuccess) return (int)e;
    const dim3 vg((unsigned)((a.np + 255) / 256 < 256 ? (a.np + 255) / 256 : 256), (unsigned)nrhs);
    k_blk_pack<<<vg, 256, 0, cs>>>(B, ldb, n, a.np, (int)nrhs, a.R, a.Y);
    const int err = launch(a, mT, mI, sms, cs);
    if (err) return err;
    k_blk_unpack<<<vg, 256, 0, cs>>>(a.Y, n, a.np, B, ldb);
    lnb_prof_count(3);
    return (int)cudaGetLastError();
}
