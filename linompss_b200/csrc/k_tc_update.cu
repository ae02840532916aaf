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
// Output tiles 128 x 128, K staged 128 bytes at a time by TMA (128B swizzle,
// no multicast), persistent CTAs (one per SM, at most 16 tiles each) walking the launch's tile list,
// two TMEM accumulators (2 x 128 columns) so the epilogue of one tile
// overlaps the mainloop of the next.  Warp roles: warp 0 lane 0 issues TMA,
// warp 1 lane 0 issues tcgen05.mma, warps 2..5 run the epilogue (tcgen05.ld
// -> registers -> C).  Every mbarrier wait is bounded; on expiry the CTA
// records a timeout, drains what it issued and frees TMEM.
#include <cuda.h>
#include <stdlib.h>

#include "tc_sm100.cuh"

namespace lnb {

enum { MODE_TF32X3 = 0, MODE_TF32 = 1, MODE_BF16 = 2 };
constexpr int64_t TC_MAX_TILES = 16;   // default tiles one CTA walks at most (see the launcher)

// LNB_TC_MAX_TILES overrides the cap (read once)
static int64_t tc_max_tiles()
{
    static int64_t v = -1;
    if (v < 0) {
        const char *e = getenv("LNB_TC_MAX_TILES");
        v = (e && atoi(e) > 0) ? atoi(e) : TC_MAX_TILES;
    }
    return v;
}

// LNB_TC_PAIR=0 selects the single-CTA 128 x 128 kernel instead of CTA pairs
// (read at every launch)
static int tc_pair()
{
    const char *e = getenv("LNB_TC_PAIR");
    return (e && *e) ? (atoi(e) != 0) : 1;
}

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

// Tiles of one launch: the lower part of a (tiles_r x tiles_c) grid of 128 x 128
// tiles whose origin is (c0, c0); tile (ti, tj) holds rows c0+128 ti.., columns
// c0+128 tj..  It is needed when it reaches r >= c, i.e. ti >= tj (square tiles,
// common origin).  Linear index l = ti (ti + 1) / 2 + tj over ti >= tj, limited to
// tj < tiles_c.
struct TileList {
    int tiles_r, tiles_c;
    int64_t count;
};

LNB_DEV void tile_of(const TileList &tl, int64_t l, int &ti, int &tj)
{
    // rows ti < tiles_c contribute ti + 1 tiles each, later rows tiles_c each
    const int64_t tri = (int64_t)tl.tiles_c * (tl.tiles_c + 1) / 2;
    if (l < tri) {
        int r = (int)((sqrt(8.0 * (double)l + 1.0) - 1.0) * 0.5);
        while ((int64_t)r * (r + 1) / 2 > l) --r;
        while ((int64_t)(r + 1) * (r + 2) / 2 <= l) ++r;
        ti = r;
        tj = (int)(l - (int64_t)r * (r + 1) / 2);
    } else {
        const int64_t q = l - tri;
        ti = tl.tiles_c + (int)(q / tl.tiles_c);
        tj = (int)(q % tl.tiles_c);
    }
}

// Persistent, warp-specialized: warp 0 = TMA producer, warp 1 = MMA issuer
// (and TMEM owner), warps 2..5 = epilogue.  TMEM holds two 128x128 fp32
// accumulators so the epilogue of one tile overlaps the mainloop of the next.
template <int MODE>
__global__ void __launch_bounds__(192, 1)
    k_tc_syrk_lower(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                    float *C, int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim, TileList tl,
                    const float *scale, lnb_status_t *st, long long wait_ns)
{
    using Cfg = TcCfg<MODE>;
    constexpr int ST = Cfg::ST;
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(sm + ST * Cfg::STAGE_BYTES);
    uint64_t *empty = full + ST;
    uint64_t *acc_full = empty + ST;      // [2]
    uint64_t *acc_empty = acc_full + 2;   // [2]
    uint32_t *tmem_slot = (uint32_t *)(acc_empty + 2);
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ktiles = (kdim + Cfg::BKE - 1) / Cfg::BKE;
    const int64_t G = gridDim.x;

    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&acc_full[a], 1);
            tc::mbar_init(&acc_empty[a], 128);
        }
        tc::fence_mbar_init();
        abort_flag = 0;
        tc::prefetch_tmap(&tm_a);
        tc::prefetch_tmap(&tm_b);
    }
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 256);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer ----------------
            int64_t kt_global = 0, issued = 0;
            for (int64_t l = blockIdx.x; l < tl.count && !abort_flag; l += G) {
                int ti, tj;
                tile_of(tl, l, ti, tj);
                const int rbase = (int)(c0 + (int64_t)ti * 128), cbase = (int)(c0 + (int64_t)tj * 128);
                for (int kt = 0; kt < ktiles; ++kt, ++kt_global) {
                    const int s = (int)(kt_global % ST);
                    const int64_t u = kt_global / ST;
                    if (kt_global >= ST && !tc::mbar_wait(&empty[s], (uint32_t)((u - 1) & 1), wait_ns, &abort_flag, st)) {
                        if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 10); }
                        break;
                    }
                    unsigned char *base = sm + s * Cfg::STAGE_BYTES;
                    tc::mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
                    const int kx = kt * Cfg::BKE;
                    if (MODE == MODE_TF32X3) {
                        tc::tma_load_2d(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, rbase);   // A hi
                        tc::tma_load_2d(base + 1 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, rbase);   // A lo
                        tc::tma_load_2d(base + 2 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, cbase);   // B hi
                        tc::tma_load_2d(base + 3 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, cbase);   // B lo
                    } else {
                        tc::tma_load_2d(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, rbase);
                        tc::tma_load_2d(base + 1 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, cbase);
                    }
                    issued = kt_global + 1;
                }
            }
            // drain: the loads still in flight must land before the CTA exits
            for (int64_t k = (issued > ST ? issued - ST : 0); k < issued; ++k)
                tc::mbar_wait(&full[k % ST], (uint32_t)((k / ST) & 1), wait_ns, &abort_flag, st);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer ----------------
            constexpr uint32_t ID = (MODE == MODE_BF16) ? tc::idesc(1, 128, 128) : tc::idesc(2, 128, 128);
            int64_t kt_global = 0;
            int lt = 0;
            for (int64_t l = blockIdx.x; l < tl.count && !abort_flag; l += G, ++lt) {
                const int acc = lt & 1;
                if (lt >= 2 && !tc::mbar_wait(&acc_empty[acc], (uint32_t)(((lt >> 1) - 1) & 1), wait_ns, &abort_flag, st)) {
                    if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 13); }
                    break;
                }
                tc::fence_after_sync();
                const uint32_t d = tmem + acc * 128;
                uint32_t accumulate = 0;
                for (int kt = 0; kt < ktiles; ++kt, ++kt_global) {
                    const int s = (int)(kt_global % ST);
                    const int64_t u = kt_global / ST;
                    if (!tc::mbar_wait(&full[s], (uint32_t)(u & 1), wait_ns, &abort_flag, st)) {
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
                            tc::mma_tf32(d, alo, bhi, ID, accumulate);
                            tc::mma_tf32(d, ahi, blo, ID, 1);
                            tc::mma_tf32(d, ahi, bhi, ID, 1);
                        } else {
                            const uint64_t am = tc::sdesc_kmajor_sw128(base + 0 * Cfg::TILE_BYTES + off);
                            const uint64_t bm = tc::sdesc_kmajor_sw128(base + 1 * Cfg::TILE_BYTES + off);
                            if (MODE == MODE_BF16) tc::mma_f16(d, am, bm, ID, accumulate);
                            else tc::mma_tf32(d, am, bm, ID, accumulate);
                        }
                        accumulate = 1;
                    }
                    tc::mma_commit(&empty[s]);      // stage s free once these MMAs have read it
                }
                tc::mma_commit(&acc_full[acc]);     // accumulator acc complete
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue warps 2..5: TMEM -> registers -> C ----------------
        const int q = warp & 3;                     // TMEM lane quarter this warp may access
        const int et = tid - 64;                    // 0..127
        int lt = 0;
        for (int64_t l = blockIdx.x; l < tl.count; l += G, ++lt) {
            int ti, tj;
            tile_of(tl, l, ti, tj);
            const int acc = lt & 1;
            const bool ok = tc::mbar_wait(&acc_full[acc], (uint32_t)((lt >> 1) & 1), wait_ns, &abort_flag, st);
            tc::fence_after_sync();
            if (!ok && !abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 12); }
            if (!__all_sync(0xffffffffu, ok && !abort_flag)) break;
            const int64_t rbase = c0 + (int64_t)ti * 128, cbase = c0 + (int64_t)tj * 128;
            const int64_t r = rbase + q * 32 + lane;
            float sr = 1.f;
            if (MODE == MODE_BF16 && r < nrows) sr = scale[r >> 7];
#pragma unroll 1
            for (int ch = 0; ch < 4; ++ch) {
                float v[32];
                tc::tmem_ld_32x32b_x32(tmem + acc * 128 + ((uint32_t)(q * 32) << 16) + ch * 32, v);
                if (r < nrows) {
                    // all 32 loads first, then the stores: loads and stores through one
                    // pointer would otherwise be serialized into 32 memory round trips
                    float cv[32];
                    float *crow = C + r + (cbase + ch * 32) * ldc;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t c = cbase + ch * 32 + j;
                        cv[j] = (c < c1 && r >= c) ? crow[(int64_t)j * ldc] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t c = cbase + ch * 32 + j;
                        if (c < c1 && r >= c) {
                            float x = v[j];
                            if (MODE == MODE_BF16) x *= sr * scale[c >> 7];
                            crow[(int64_t)j * ldc] = cv[j] - x;
                        }
                    }
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&acc_empty[acc]);       // 128 arrivals release the accumulator
            (void)et;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 1) tc::tmem_dealloc(tmem, 256);
}

// ---- CTA-pair variant ---------------------------------------------------------
// A 2-CTA cluster computes 256 x 256 tiles with cta_group::2 MMAs (M = N = 256).
// CTA r loads rows [128 r, 128 r + 128) of the tile's A rows and of its B
// (column) rows, holds rows [128 r, 128 r + 128) x all 256 columns of the
// accumulator in its TMEM and writes them back; rank 0 issues the MMAs and
// multicasts their completion to both CTAs.  Per SM this halves the operand
// bytes per flop of the single-CTA 128 x 128 tile, so the same pipeline depth
// hides twice the load latency.  Eight epilogue warps (two per TMEM lane
// quarter) drain the 128 x 256 accumulator.
template <int MODE>
struct Tc2Cfg {
    static constexpr int TILE_BYTES = 128 * 128;                   // one 128-row x 128-byte operand box
    static constexpr int NT = (MODE == MODE_TF32X3) ? 4 : 2;       // boxes per stage per CTA
    static constexpr int STAGE_BYTES = NT * TILE_BYTES;
    static constexpr int ST = (MODE == MODE_TF32X3) ? 3 : 6;
    static constexpr int BKE = (MODE == MODE_BF16) ? 64 : 32;
    static constexpr int KSTEP_BYTES = 32;
    static constexpr int EPI_WARPS = 8;
    static constexpr int THREADS = 64 + 32 * EPI_WARPS;           // producer, MMA issuer, epilogue
    static constexpr int SMEM = ST * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
};

template <int MODE>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Tc2Cfg<MODE>::THREADS, 1)
    k_tc2_syrk_lower(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b, float *C,
                     int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim, TileList tl, const float *scale,
                     lnb_status_t *st, long long wait_ns)
{
    using Cfg = Tc2Cfg<MODE>;
    constexpr int ST = Cfg::ST;
    extern __shared__ __align__(1024) unsigned char smraw[];
    unsigned char *sm = (unsigned char *)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(sm + ST * Cfg::STAGE_BYTES);   // rank 0's count both CTAs' loads
    uint64_t *empty = full + ST;
    uint64_t *acc_full = empty + ST;      // [2]
    uint64_t *acc_empty = acc_full + 2;   // [2], rank 0's: every epilogue warp of both CTAs
    uint32_t *tmem_slot = (uint32_t *)(acc_empty + 2);
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = tc::cluster_rank();
    const int ktiles = (kdim + Cfg::BKE - 1) / Cfg::BKE;
    const int64_t G = gridDim.x / 2, pair = blockIdx.x / 2;

    if (tid == 0) {
        for (int s = 0; s < ST; ++s) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&acc_full[a], 1);
            tc::mbar_init(&acc_empty[a], 2 * Cfg::EPI_WARPS);
        }
        tc::fence_mbar_init();
        abort_flag = 0;
        tc::prefetch_tmap(&tm_a);
        tc::prefetch_tmap(&tm_b);
    }
    if (warp == 1) {
        tc::tmem_alloc2(tmem_slot, 512);
        tc::tmem_relinquish2();
    }
    tc::fence_before_sync();
    tc::cluster_sync();                   // both CTAs' barriers and the TMEM address are in place
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer (both CTAs) ----------------
            int64_t kt_global = 0, issued = 0;
            for (int64_t l = pair; l < tl.count && !abort_flag; l += G) {
                int ti, tj;
                tile_of(tl, l, ti, tj);
                const int arow = (int)(c0 + (int64_t)ti * 256 + rank * 128);
                const int brow = (int)(c0 + (int64_t)tj * 256 + rank * 128);
                for (int kt = 0; kt < ktiles; ++kt, ++kt_global) {
                    const int s = (int)(kt_global % ST);
                    const int64_t u = kt_global / ST;
                    if (kt_global >= ST && !tc::mbar_wait(&empty[s], (uint32_t)((u - 1) & 1), wait_ns, &abort_flag, st)) {
                        if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 20); }
                        break;
                    }
                    unsigned char *base = sm + s * Cfg::STAGE_BYTES;
                    if (rank == 0) tc::mbar_arrive_expect_tx(&full[s], 2 * Cfg::STAGE_BYTES);
                    const int kx = kt * Cfg::BKE;
                    if (MODE == MODE_TF32X3) {
                        tc::tma_load_2d_pair(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, arow);   // A hi
                        tc::tma_load_2d_pair(base + 1 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, arow);   // A lo
                        tc::tma_load_2d_pair(base + 2 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, brow);   // B hi
                        tc::tma_load_2d_pair(base + 3 * Cfg::TILE_BYTES, &tm_b, &full[s], kx, brow);   // B lo
                    } else {
                        tc::tma_load_2d_pair(base + 0 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, arow);
                        tc::tma_load_2d_pair(base + 1 * Cfg::TILE_BYTES, &tm_a, &full[s], kx, brow);
                    }
                    issued = kt_global + 1;
                }
            }
            // rank 0's barriers count both CTAs' loads: it drains the ones in flight
            if (rank == 0)
                for (int64_t k = (issued > ST ? issued - ST : 0); k < issued; ++k)
                    tc::mbar_wait(&full[k % ST], (uint32_t)((k / ST) & 1), wait_ns, &abort_flag, st);
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0 && rank == 0) {
            // ---------------- MMA issuer (rank 0) ----------------
            constexpr uint32_t ID = (MODE == MODE_BF16) ? tc::idesc(1, 256, 256) : tc::idesc(2, 256, 256);
            int64_t kt_global = 0;
            int lt = 0;
            for (int64_t l = pair; l < tl.count && !abort_flag; l += G, ++lt) {
                const int acc = lt & 1;
                if (lt >= 2 && !tc::mbar_wait(&acc_empty[acc], (uint32_t)(((lt >> 1) - 1) & 1), wait_ns, &abort_flag, st)) {
                    if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 23); }
                    break;
                }
                tc::fence_after_sync();
                const uint32_t d = tmem + acc * 256;
                uint32_t accumulate = 0;
                for (int kt = 0; kt < ktiles; ++kt, ++kt_global) {
                    const int s = (int)(kt_global % ST);
                    const int64_t u = kt_global / ST;
                    if (!tc::mbar_wait(&full[s], (uint32_t)(u & 1), wait_ns, &abort_flag, st)) {
                        if (!abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 21); }
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
                            tc::mma2_tf32(d, alo, bhi, ID, accumulate);
                            tc::mma2_tf32(d, ahi, blo, ID, 1);
                            tc::mma2_tf32(d, ahi, bhi, ID, 1);
                        } else {
                            const uint64_t am = tc::sdesc_kmajor_sw128(base + 0 * Cfg::TILE_BYTES + off);
                            const uint64_t bm = tc::sdesc_kmajor_sw128(base + 1 * Cfg::TILE_BYTES + off);
                            if (MODE == MODE_BF16) tc::mma2_f16(d, am, bm, ID, accumulate);
                            else tc::mma2_tf32(d, am, bm, ID, accumulate);
                        }
                        accumulate = 1;
                    }
                    tc::mma2_commit_mc(&empty[s], 0x3);    // stage s free in both CTAs
                }
                tc::mma2_commit_mc(&acc_full[acc], 0x3);   // accumulator acc complete in both CTAs
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue warps 2..9 (both CTAs): TMEM -> registers -> C ----------------
        const int q = warp & 3;                 // TMEM lane quarter this warp may access
        const int h = (warp - 2) >> 2;          // column half: chunks [4 h, 4 h + 4)
        int lt = 0;
        for (int64_t l = pair; l < tl.count; l += G, ++lt) {
            int ti, tj;
            tile_of(tl, l, ti, tj);
            const int acc = lt & 1;
            const bool ok = tc::mbar_wait(&acc_full[acc], (uint32_t)((lt >> 1) & 1), wait_ns, &abort_flag, st);
            tc::fence_after_sync();
            if (!ok && !abort_flag) { abort_flag = 1; atomicCAS(&st->timeout, 0, 22); }
            if (!__all_sync(0xffffffffu, ok && !abort_flag)) break;
            const int64_t rbase = c0 + (int64_t)ti * 256 + rank * 128, cbase = c0 + (int64_t)tj * 256;
            const int64_t r = rbase + q * 32 + lane;
            float sr = 1.f;
            if (MODE == MODE_BF16 && r < nrows) sr = scale[r >> 7];
#pragma unroll 1
            for (int ch = 4 * h; ch < 4 * h + 4; ++ch) {
                float v[32];
                tc::tmem_ld_32x32b_x32(tmem + acc * 256 + ((uint32_t)(q * 32) << 16) + ch * 32, v);
                if (r < nrows) {
                    float cv[32];
                    float *crow = C + r + (cbase + ch * 32) * ldc;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t c = cbase + ch * 32 + j;
                        cv[j] = (c < c1 && r >= c) ? crow[(int64_t)j * ldc] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int64_t c = cbase + ch * 32 + j;
                        if (c < c1 && r >= c) {
                            float x = v[j];
                            if (MODE == MODE_BF16) x *= sr * scale[c >> 7];
                            crow[(int64_t)j * ldc] = cv[j] - x;
                        }
                    }
                }
            }
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive_remote(&acc_empty[acc], 0);   // releases the accumulator to rank 0
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::cluster_sync();                   // no pair MMA or remote arrival still targets this CTA
    if (warp == 1) tc::tmem_dealloc2(tmem, 512);
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

// K-major operand copy: rows x kext elements, row stride kstride elements, box
// 128 rows x 128 bytes; K beyond kext reads as zero
static int make_map(CUtensorMap *m, const void *base, int64_t rows, int kext, int64_t kstride, bool bf16)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return (int)cudaErrorNotSupported;
    const int esz = bf16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)kext, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kstride * esz};
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

// mode: 0 = TF32x3 (hi, lo), 1 = TF32 (hi), 2 = BF16 (hi = bf16 copy, scale).
// The operands are K-major with row stride kstride (elements, a multiple of
// 16 bytes); the first kdim K columns are used.
extern "C" int lnb_k_tc_syrk_lower(int mode, const void *hi, const void *lo, int64_t kstride, int64_t prow, float *C,
                                   int64_t ldc, int64_t nrows, int64_t c0, int64_t c1, int kdim, const float *scale,
                                   lnb_status_t *st, long long wait_ns, lnb_stream_t s)
{
    if (nrows <= c0 || c1 <= c0 || kdim <= 0) return 0;
    if ((uintptr_t)hi % 16 || (lo && (uintptr_t)lo % 16)) return (int)cudaErrorMisalignedAddress;
    CUtensorMap ta, tb;
    int e = make_map(&ta, hi, prow, kdim, kstride, mode == MODE_BF16);
    if (!e) e = make_map(&tb, mode == MODE_TF32X3 ? lo : hi, prow, kdim, kstride, mode == MODE_BF16);
    if (e) return e;
    TileList tl;
    tl.tiles_c = (int)((c1 - c0 + 127) / 128);
    tl.tiles_r = (int)((nrows - c0 + 127) / 128);
    {
        const int64_t tc_ = tl.tiles_c, tr_ = tl.tiles_r;
        const int64_t m = tc_ < tr_ ? tc_ : tr_;
        tl.count = m * (m + 1) / 2 + (tr_ > tc_ ? (tr_ - tc_) * tc_ : 0);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (tc_pair()) {
        // 256 x 256 tiles on CTA pairs
        TileList t2;
        t2.tiles_c = (int)((c1 - c0 + 255) / 256);
        t2.tiles_r = (int)((nrows - c0 + 255) / 256);
        {
            const int64_t tc_ = t2.tiles_c, tr_ = t2.tiles_r;
            const int64_t m = tc_ < tr_ ? tc_ : tr_;
            t2.count = m * (m + 1) / 2 + (tr_ > tc_ ? (tr_ - tc_) * tc_ : 0);
        }
        int64_t pairs = t2.count < sms / 2 ? t2.count : sms / 2;
        int64_t mt2 = tc_max_tiles() * 512 / (4 * (int64_t)kdim);   // a pair tile is four 128 x 128 tiles
        if (mt2 < 1) mt2 = 1;
        const int64_t pcap = (t2.count + mt2 - 1) / mt2;
        // more pairs than fit at once: whole waves, so that no pair runs its
        // tiles after all the others have finished
        const int64_t slots = sms / 2;
        if (pcap > pairs) pairs = (pcap + slots - 1) / slots * slots;
        if (pairs > t2.count) pairs = t2.count;
        dim3 grid2((unsigned)(2 * pairs));
        switch (mode) {
        case MODE_TF32X3:
            cudaFuncSetAttribute(k_tc2_syrk_lower<MODE_TF32X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Tc2Cfg<MODE_TF32X3>::SMEM);
            k_tc2_syrk_lower<MODE_TF32X3><<<grid2, Tc2Cfg<MODE_TF32X3>::THREADS, Tc2Cfg<MODE_TF32X3>::SMEM, s>>>(
                ta, tb, C, ldc, nrows, c0, c1, kdim, t2, scale, st, wait_ns);
            break;
        case MODE_TF32:
            cudaFuncSetAttribute(k_tc2_syrk_lower<MODE_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Tc2Cfg<MODE_TF32>::SMEM);
            k_tc2_syrk_lower<MODE_TF32><<<grid2, Tc2Cfg<MODE_TF32>::THREADS, Tc2Cfg<MODE_TF32>::SMEM, s>>>(
                ta, tb, C, ldc, nrows, c0, c1, kdim, t2, scale, st, wait_ns);
            break;
        default:
            cudaFuncSetAttribute(k_tc2_syrk_lower<MODE_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Tc2Cfg<MODE_BF16>::SMEM);
            k_tc2_syrk_lower<MODE_BF16><<<grid2, Tc2Cfg<MODE_BF16>::THREADS, Tc2Cfg<MODE_BF16>::SMEM, s>>>(
                ta, tb, C, ldc, nrows, c0, c1, kdim, t2, scale, st, wait_ns);
            break;
        }
        lnb_prof_count(1);
        return (int)cudaGetLastError();
    }
    // persistent, but a CTA walks at most TC_MAX_TILES tiles: long updates then
    // retire CTAs every few hundred microseconds, which lets the high-priority
    // stream's panel kernels (POTRF, TRSM) take SMs in the middle of an update
    int64_t g = tl.count < sms ? tl.count : sms;
    // the cap counts 512-deep tiles: a CTA of a long-K update walks fewer
    int64_t mt = tc_max_tiles() * 512 / kdim;
    if (mt < 1) mt = 1;
    const int64_t gcap = (tl.count + mt - 1) / mt;
    if (gcap > g) g = (gcap + sms - 1) / sms * sms;   // whole waves
    if (g > tl.count) g = tl.count;
    dim3 grid((unsigned)g);
    switch (mode) {
    case MODE_TF32X3:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_TF32X3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_TF32X3>::SMEM);
        k_tc_syrk_lower<MODE_TF32X3><<<grid, 192, TcCfg<MODE_TF32X3>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1,
                                                                                kdim, tl, scale, st, wait_ns);
        break;
    case MODE_TF32:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_TF32>::SMEM);
        k_tc_syrk_lower<MODE_TF32><<<grid, 192, TcCfg<MODE_TF32>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1, kdim,
                                                                            tl, scale, st, wait_ns);
        break;
    default:
        cudaFuncSetAttribute(k_tc_syrk_lower<MODE_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TcCfg<MODE_BF16>::SMEM);
        k_tc_syrk_lower<MODE_BF16><<<grid, 192, TcCfg<MODE_BF16>::SMEM, s>>>(ta, tb, C, ldc, nrows, c0, c1, kdim,
                                                                            tl, scale, st, wait_ns);
        break;
    }
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
