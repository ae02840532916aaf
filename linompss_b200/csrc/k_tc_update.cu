// k_tc_update.cu -- low-precision trailing update on the 5th-generation tensor
// cores: C[r,c] -= sum_k P[r,k] P[c,k] for r >= c (the SYRK and GEMM tile
// tasks of one k-step, chol_rlmain.c:40-49, fused), C in FP32.
//
// Operands are K-major copies of the solved panel made by k_prep_* :
//   MODE_TF32X3 : P = hi + lo (hi = rna_tf32(P)); three kind::tf32 MMAs per
//                 K step, hi*hi + hi*lo + lo*hi, FP32 accumulation in TMEM:
//                 ~FP32-accurate products at tensor-core rate
//   MODE_TF32   : one kind::tf32 MMA (hi*hi)
//   MODE_BF16   : P = s_blk * bf16(P / s_blk) with a power-of-two scale per
//                 128-row block; one kind::f16 MMA, epilogue multiplies by
//                 s_i * s_j
// CTA tile 128 x 128, K staged 128 bytes at a time by TMA (128B swizzle, no
// multicast), accumulator in TMEM (128 columns).  Warp roles: warp 0 lane 0
// issues TMA, warp 1 lane 0 issues tcgen05.mma, all four warps run the
// epilogue (tcgen05.ld -> registers -> C).  Every mbarrier wait is bounded;
// on expiry the CTA records a timeout, drains what it issued and frees TMEM.
#include <cuda.h>

#include "tc_sm100.cuh"

namespace lnb {

enum { MODE_TF32X3 = 0, MODE_TF32 = 1, MODE_BF16 = 2 };

template <int MODE>
struct TcCfg {
    static constexpr int BM = 128, BN = 128;
    static constexpr int TILE_BYTES = 128 * 128;                   // one 128-row x 128-byte operand tile
    static constexpr int NT = (MODE == MODE_TF32X3) ? 4 : 2;       // operand tiles per stage
    static constexpr int STAGE_BYTES = NT * TILE_BYTES;
    static constexpr int ST = (MODE == MODE_TF32X3) ? 3 : 6;
    static constexpr int BKE = (MODE == MODE_BF16) ? 64 : 32;      // K elements per stage
    static constexpr int KSTEP_BYTES = 32;                          // K of one MMA = 32 bytes
    static constexpr int SMEM = ST * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
};

template <int MODE>
__global__ void __launch_bounds__(128, 1)
    k_tc_syrk_lower(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                    float *C, int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim,
                    const float *scale, lnb_status_t *st, long long wait_ns)
{
    using Cfg = TcCfg<MODE>;
    constexpr int ST = Cfg::ST;
    const int tj = blockIdx.x, ti = blockIdx.y;
    const int64_t rbase = c0 + (int64_t)ti * Cfg::BM, cbase = c0 + (int64_t)tj * Cfg::BN;
    if (rbase + Cfg::BM <= cbase || rbase >= nrows || cbase >= c1) return;

    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(sm + ST * Cfg::STAGE_BYTES);
    uint64_t *empty = full + ST;
    uint64_t *accb = empty + ST;
    uint32_t *tmem_slot = (uint32_t *)(accb + 1);
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ktiles = (kdim + Cfg::BKE - 1) / Cfg::BKE;

    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        tc::mbar_init(accb, 1);
        tc::fence_mbar_init();
        abort_flag = 0;
        tc::prefetch_tmap(&tm_a);
        tc::prefetch_tmap(&tm_b);
    }
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, 128);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (tid == 0) {
        // ---------------- TMA producer ----------------
        int issued = 0;
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % ST, u = kt / ST;
            if (kt >= ST && !tc::mbar_wait(&empty[s], (u - 1) & 1, wait_ns, &abort_flag, st)) {
                if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 10); }
                break;
            }
            unsigned char *base = sm + s * Cfg::STAGE_BYTES;
            tc::mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
            const int kx = kt * Cfg::BKE;
            if (MODE == MODE_TF32X3) {
                tc::tma_load_2d(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, (int)rbase);   // A hi
                tc::tma_load_2d(base + 1 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, (int)rbase);   // A lo
                tc::tma_load_2d(base + 2 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, (int)cbase);   // B hi
                tc::tma_load_2d(base + 3 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, (int)cbase);   // B lo
            } else {
                tc::tma_load_2d(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, (int)rbase);
                tc::tma_load_2d(base + 1 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, (int)cbase);
            }
            issued = kt + 1;
        }
        // drain: every stage load issued must land before the CTA can exit
        for (int kt = (issued > ST ? issued - ST : 0); kt < issued; ++kt)
            tc::mbar_wait(&full[kt % ST], (kt / ST) & 1, wait_ns, &abort_flag, st);
    } else if (tid == 32) {
        // ---------------- MMA issuer ----------------
        constexpr uint32_t ID = (MODE == MODE_BF16) ? tc::idesc(1, 128, 128) : tc::idesc(2, 128, 128);
        uint32_t accumulate = 0;
        for (int kt = 0; kt < ktiles; ++kt) {
            const int s = kt % ST, u = kt / ST;
            if (!tc::mbar_wait(&full[s], u & 1, wait_ns, &abort_flag, st)) {
                if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 11); }
                break;
            }
            tc::fence_after_sync();
            const uint32_t base = smem_u32(sm + s * Cfg::STAGE_BYTES);
#pragma unroll
            for (int kk = 0; kk < 128 / Cfg::KSTEP_BYTES; ++kk) {
                const uint32_t off = kk * Cfg::KSTEP_BYTES;
                if (MODE == MODE_TF32X3) {
                    const uint64_t ahi = tc::sdesc_kmajor_sw128(base + 0 * Cfg::TILE_BYTES + off);
                    const uint64_t alo = tc::sdesc_kmajor_sw128(base + 1 * Cfg::TILE_BYTES + off);
                    const uint64_t bhi = tc::sdesc_kmajor_sw128(base + 2 * Cfg::TILE_BYTES + off);
                    const uint64_t blo = tc::sdesc_kmajor_sw128(base + 3 * Cfg::TILE_BYTES + off);
                    tc::mma_tf32(tmem, alo, bhi, ID, accumulate);
                    tc::mma_tf32(tmem, ahi, blo, ID, 1);
                    tc::mma_tf32(tmem, ahi, bhi, ID, 1);
                } else {
                    const uint64_t a = tc::sdesc_kmajor_sw128(base + 0 * Cfg::TILE_BYTES + off);
                    const uint64_t b = tc::sdesc_kmajor_sw128(base + 1 * Cfg::TILE_BYTES + off);
                    if (MODE == MODE_BF16) tc::mma_f16(tmem, a, b, ID, accumulate);
                    else tc::mma_tf32(tmem, a, b, ID, accumulate);
                }
                accumulate = 1;
            }
            tc::mma_commit(&empty[s]);     // stage s free once these MMAs have read it
        }
        tc::mma_commit(accb);              // accumulator complete (covers every MMA issued)
    }
    __syncwarp();

    // ---------------- epilogue: TMEM -> registers -> C ----------------
    const bool ok = tc::mbar_wait(accb, 0, wait_ns, &abort_flag, st);
    tc::fence_after_sync();
    if (!ok && !abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 12); }
    // tcgen05.ld is warp-collective: the whole warp takes the same branch
    const bool do_epi = __all_sync(0xffffffffu, ok && !abort_flag);
    if (do_epi) {
        const int64_t r = rbase + warp * 32 + lane;
        float sr = 1.f;
        if (MODE == MODE_BF16 && r < nrows) sr = scale[r >> 7];
#pragma unroll 1
        for (int ch = 0; ch < Cfg::BN / 32; ++ch) {
            float v[32];
            tc::tmem_ld_32x32b_x32(tmem + ((uint32_t)(warp * 32) << 16) + ch * 32, v);
            if (r < nrows) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int64_t c = cbase + ch * 32 + j;
                    if (c < c1 && r >= c) {
                        float x = v[j];
                        if (MODE == MODE_BF16) x *= sr * scale[c >> 7];
                        C[r + c * ldc] -= x;
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

// ---- host: tensor maps ---------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// K-major operand copy: rows x kpad elements (row stride kpad), box 128 rows x 128 bytes
static int make_map(CUtensorMap *m, const void *base, int64_t rows, int kpad, bool bf16)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return (int)cudaErrorNotSupported;
    const int esz = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kpad * esz};
    cuuint32_t box[2] = {(cuuint32_t)(128 / esz), 128};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                    const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)cudaErrorInvalidValue;
}

}  // namespace lnb

using namespace lnb;

// mode: 0 = TF32x3 (hi, lo), 1 = TF32 (hi), 2 = BF16 (hi = bf16 copy, scale)
extern "C" int lnb_k_tc_syrk_lower(int mode, const void *hi, const void *lo, int kpad, int64_t prow, float *C,
                                   int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim, const float *scale,
                                   lnb_status_t *st, long long wait_ns, lnb_stream_t s)
{
    if (nrows <= c0 || c1 <= c0 || kdim <= 0) return 0;
    if ((uintptr_t)hi % 16 || (lo && (uintptr_t)lo % 16)) return (int)cudaErrorMisalignedAddress;
    CUtensorMap ta, tb;
    int e = make_map(&ta, hi, prow, kpad, mode == MODE_BF16);
    if (!e) e = make_map(&tb, mode == MODE_TF32X3 ? lo : hi, prow, kpad, mode == MODE_BF16);
    if (e) return e;
    dim3 grid((unsigned)((c1 - c0 + 127) / 128), (unsigned)((nrows - c0 + 127) / 128));
    switch (mode) {
    case MODE_TF32X3:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_TF32X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_TF32X3>::SMEM);
        k_tc_syrk_lower<MODE_TF32X3><<<grid, 128, TcCfg<MODE_TF32X3>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1,
                                                                                kdim, scale, st, wait_ns);
        break;
    case MODE_TF32:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_TF32>::SMEM);
        k_tc_syrk_lower<MODE_TF32><<<grid, 128, TcCfg<MODE_TF32>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1, kdim,
                                                                            scale, st, wait_ns);
        break;
    default:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_BF16>::SMEM);
        k_tc_syrk_lower<MODE_BF16><<<grid, 128, TcCfg<MODE_BF16>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1, kdim,
                                                                            scale, st, wait_ns);
        break;
    }
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
