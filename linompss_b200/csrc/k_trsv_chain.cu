// k_trsv_chain.cu -- blocked triangular solves with few right-hand sides
// (nrhs <= 8): op(T) X = B, T triangular, FP64 arithmetic on FP64 or FP32 T.
//
// Semantics of bblas_dltrsm (bblas_trsm.h:116-202) and of the two solves of
// dspdsolv_main (spdsolv_main.c:15,17), as k_trsv.cu.  With one or a few
// right-hand sides the solve is a chain of nb = n/64 dependent diagonal
// steps with O(n^2) independent work hanging off it, so the launch is
// organised around the chain:
//
//   * one CTA (the first to draw a ticket) walks the chain.  Its 8 compute
//     warps keep the last W solution blocks in shared memory and apply the W
//     sub-diagonal tiles of each block row themselves, so no global-memory
//     round trip sits between two chain steps.  The W band tiles of the next
//     step stream in by cp.async while the current step computes (from L2:
//     they and the diagonal inverses are bulk-prefetched PF steps ahead), and
//     the inverse of the next diagonal block streams into registers.
//   * a loader warp of the same CTA (4 lane groups, one upcoming block row
//     each) waits until the far-off-diagonal updates of a row are complete
//     and stages its right-hand sides into shared memory with cp.async ahead
//     of the compute warps;
//   * a publisher warp makes finished solution blocks visible to the whole
//     GPU (one release fence for all blocks finished so far, then their
//     flags) off the compute warps' path;
//   * every other CTA takes work items (row i, a chunk of CW tiles j <=
//     i-W-1) from an atomic ticket in row order.  An item streams its tiles
//     (double-buffered across items) before it waits for its solution blocks,
//     then subtracts op(T)_ij X_j from B_i with atomics and bumps the row's
//     counter.  Items of row i only wait on blocks j < i-W, which the chain
//     produced before it needs row i, so the walk cannot deadlock.
// Every wait is bounded and reports a site code in the status word.
#include <stdlib.h>
#include <string.h>

#include "common.cuh"
#include "tc_sm100.cuh"

namespace lnb {
namespace chain {

constexpr int TH = 64;              // block size
constexpr int NCOMP = 256;          // compute threads: m = t>>2, kq = t&3
constexpr int NTHR = NCOMP + 64;    // + publisher warp + loader warp
constexpr int NBUF = 4;             // right-hand-side slots = loader lane groups
constexpr int XR = 4;               // finished-block slots between compute and publisher
constexpr int PF = 4;               // L2 prefetch distance of the chain, in steps

// band width W handled by the chain CTA, worker chunk CW (tiles per item)
template <typename TT> struct Cfg;
template <> struct Cfg<float> { static constexpr int W = 4, CW = 4; };
template <> struct Cfg<double> { static constexpr int W = 2, CW = 2; };

// Padded leading dimension of a staged 64 x 64 tile S[col * LD + row].
// TR (op = transpose) reads rows of S with 16-byte vectors, 2 columns per
// 8-lane phase: LD == 16 words mod 32.  !TR reads 4 columns x 8 rows per
// phase (scalar): LD == 8 floats mod 32, or 4 doubles mod 16.
template <typename TT, bool TR> struct Ld;
template <> struct Ld<float, true> { static constexpr int v = 80; };
template <> struct Ld<float, false> { static constexpr int v = 72; };
template <> struct Ld<double, true> { static constexpr int v = 72; };
template <> struct Ld<double, false> { static constexpr int v = 68; };

template <typename TT>
struct Args {
    const TT *T; int64_t ldt; const TT *dinv;   // inverses stored in the precision of T
    double *B; int64_t ldb; int64_t n; int nrhs;
    int nb, fwd, vec;           // vec: T and ldt allow 16-byte copies
    int tma;                    // the chain CTA stages its band tiles through the tensor map (FP32)
    int *ticket, *cnt, *ready;  // cnt/ready indexed by chain position
    lnb_status_t *st; long long wait_ns;
};

LNB_DEV void cp_async4(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem)), "l"(gmem));
}
LNB_DEV void cp_async_el(float *d, const float *g) { cp_async4(d, g); }
LNB_DEV void cp_async_el(double *d, const double *g) { cp_async8(d, g, true); }

// 16-byte cp.async from L2 (.cg) copying src_bytes (0, 8 or 16) and zero-filling the rest
LNB_DEV void cp_async16_n(void *smem, const void *gmem, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
                 "r"(src_bytes));
}
// arrive on `bar` once this thread's earlier cp.async copies have landed
LNB_DEV void cp_async_mbar_arrive(uint64_t *bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from
// global to shared memory, counted on `bar`'s transaction count
LNB_DEV void bulk_copy_g2s(void *smem, const void *gmem, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem)),
                 "l"(gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// hint: bring the box at (x, y) of a tensor map into L2
LNB_DEV void prefetch_box_l2(const CUtensorMap *map, int x, int y)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global [%0, {%1, %2}];" ::"l"(map), "r"(x), "r"(y) : "memory");
}
// hint: bring `bytes` (a multiple of 16, 16-byte aligned) into L2
LNB_DEV void prefetch_l2(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
// release fence at GPU scope: orders this thread's earlier writes, and those it
// has observed through a barrier, before its later writes (cumulative)
LNB_DEV void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
LNB_DEV void st_relaxed(int *p, int v)
{
    asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// named barrier over `count` threads that also ANDs a predicate
LNB_DEV bool bar_and(int id, int count, bool pred)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

template <typename TT>
LNB_DEV int blen(const Args<TT> &a, int i)
{
    const int64_t o = (int64_t)i * TH;
    return (int)((a.n - o) < TH ? (a.n - o) : TH);
}
// actual block index of chain position p
template <typename TT>
LNB_DEV int blk(const Args<TT> &a, int p) { return a.fwd ? p : a.nb - 1 - p; }

// Stage the stored block holding op(T)(i, j) as S[col * LD + row], zero
// outside the matrix; cp.async, caller commits.
template <typename TT, bool TR>
LNB_DEV void stage_tile(const Args<TT> &a, TT *S, int i, int j, int tid, int nthr)
{
    constexpr int LD = Ld<TT, TR>::v;
    constexpr int EPC = 16 / (int)sizeof(TT);
    constexpr int CPC = TH / EPC;
    const int rb = TR ? j : i, cb = TR ? i : j;
    const int rows = blen(a, rb), cols = blen(a, cb);
    const TT *src = a.T + (int64_t)rb * TH + (int64_t)cb * TH * a.ldt;
    for (int idx = tid; idx < TH * CPC; idx += nthr) {
        const int col = idx / CPC, r = (idx % CPC) * EPC;
        TT *d = S + col * LD + r;
        const TT *g = src + r + (int64_t)col * a.ldt;
        if (col >= cols || r >= rows) {
            cp_async16(d, a.T, false);
        } else if (a.vec && r + EPC <= rows) {
            cp_async16(d, g, true);
        } else {
#pragma unroll
            for (int e = 0; e < EPC; ++e) {
                if (r + e < rows) cp_async_el(d + e, g + e);
                else d[e] = (TT)0;
            }
        }
    }
}

// L2 prefetch of column `col` of the stored block holding op(T)(i, j)
template <typename TT, bool TR>
LNB_DEV void prefetch_tile_col(const Args<TT> &a, int i, int j, int col)
{
    const int rb = TR ? j : i, cb = TR ? i : j;
    if (col >= blen(a, cb)) return;
    const uint32_t bytes = (uint32_t)(blen(a, rb) * (int)sizeof(TT)) & ~15u;
    if (bytes) prefetch_l2(a.T + (int64_t)rb * TH + ((int64_t)cb * TH + col) * a.ldt, bytes);
}

// part[r] += sum over this lane's 16 k of op[m][k] * X[r * 64 + k]
template <typename TT, int NR, bool TR>
LNB_DEV void gemv_tile(const TT *S, const double *X, int m, int kq, double (&part)[NR])
{
    constexpr int LD = Ld<TT, TR>::v;
    if constexpr (TR) {
        constexpr int EPC = 16 / (int)sizeof(TT);
#pragma unroll
        for (int u = 0; u < 16 / EPC; ++u) {
            const int k0 = EPC * (kq + 4 * u);
            TT v[EPC];
            if constexpr (EPC == 4) {
                const float4 q = *reinterpret_cast<const float4 *>(S + m * LD + k0);
                v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
            } else {
                const double2 q = *reinterpret_cast<const double2 *>(S + m * LD + k0);
                v[0] = q.x; v[1] = q.y;
            }
#pragma unroll
            for (int e = 0; e < EPC; ++e)
#pragma unroll
                for (int r = 0; r < NR; ++r) part[r] = fma((double)v[e], X[r * TH + k0 + e], part[r]);
        }
    } else {
#pragma unroll
        for (int v = 0; v < 16; ++v) {
            const int k = kq + 4 * v;
            const double t = (double)S[k * LD + m];
#pragma unroll
            for (int r = 0; r < NR; ++r) part[r] = fma(t, X[r * TH + k], part[r]);
        }
    }
}

// A 64 x 64 FP32 tile staged by TMA as two 32-row boxes (64 columns of 128
// bytes each) in the 128-byte-swizzled layout: element (row r, column c) of
// the stored block.  Needs a 1024-byte-aligned tile.
LNB_DEV int swz(int r, int c) { return ((r >> 5) << 11) + (c << 5) + ((((r & 31) >> 2) ^ (c & 7)) << 2) + (r & 3); }

// gemv_tile for a tile in that layout (FP32)
template <int NR, bool TR>
LNB_DEV void gemv_tile_sw(const float *S, const double *X, int m, int kq, double (&part)[NR])
{
    if constexpr (TR) {
        // op[m][k] = stored (row k, column m); rows k0..k0+3 are one 16-byte chunk
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k0 = 4 * (kq + 4 * u);
            const float4 q = *reinterpret_cast<const float4 *>(S + swz(k0, m));
            const float v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
#pragma unroll
                for (int r = 0; r < NR; ++r) part[r] = fma((double)v[e], X[r * TH + k0 + e], part[r]);
        }
    } else {
        // op[m][k] = stored (row m, column k)
#pragma unroll
        for (int v = 0; v < 16; ++v) {
            const int k = kq + 4 * v;
            const double t = (double)S[swz(m, k)];
#pragma unroll
            for (int r = 0; r < NR; ++r) part[r] = fma(t, X[r * TH + k], part[r]);
        }
    }
}

// k owned by lane kq for the j-th inverse element (same partition as the
// FP64 tiles, so the reads of the staged vector are conflict-free)
template <bool TR>
LNB_DEV int kd(int kq, int j) { return TR ? 2 * (kq + 4 * (j >> 1)) + (j & 1) : kq + 4 * j; }

// inverse of op(T) on diagonal block i, this lane's 16 entries of row m, kept
// in the precision of T: a conversion here would wait for each load, while the
// raw values are first needed a step later
template <bool TR, typename DT>
LNB_DEV void load_dinv(const DT *dinv, int i, int m, int kq, DT (&dv)[16])
{
    const DT *D = dinv + (int64_t)i * TH * TH;   // inv(T_ii), column-major
    if constexpr (TR) {
        // inv(T_ii^T)[m][k] = D[k + 64 m], pairs of consecutive k
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if constexpr (sizeof(DT) == 8) {
                const double2 q = __ldg(reinterpret_cast<const double2 *>(D + TH * m + 2 * (kq + 4 * u)));
                dv[2 * u] = q.x; dv[2 * u + 1] = q.y;
            } else {
                const float2 q = __ldg(reinterpret_cast<const float2 *>(D + TH * m + 2 * (kq + 4 * u)));
                dv[2 * u] = q.x; dv[2 * u + 1] = q.y;
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) dv[j] = __ldg(D + m + TH * kd<false>(kq, j));
    }
}

template <int NR>
LNB_DEV void quad_sum(double (&p)[NR])
{
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        p[r] += __shfl_xor_sync(0xffffffffu, p[r], 1);
        p[r] += __shfl_xor_sync(0xffffffffu, p[r], 2);
    }
}

// ---- worker items ------------------------------------------------------------
// Row (chain position) p holds need(p) = ceil(max(0, p - W) / CW) items;
// F(p) = sum_{q<p} need(q) = G(p - 1 - W), G(S) = sum_{s=1..S} ceil(s/CW).
template <int W, int CW>
LNB_DEV int64_t items_before(int p)
{
    const int64_t S = (int64_t)p - 1 - W;
    if (S <= 0) return 0;
    const int64_t q = S / CW, b = S % CW;
    return CW * q * (q + 1) / 2 + b * (q + 1);
}
template <int W, int CW>
LNB_DEV int need_of(int p) { return p > W ? (p - W + CW - 1) / CW : 0; }

template <int W, int CW>
LNB_DEV void decode(int64_t q, int nb, int &row, int &chunk)
{
    int lo = 0, hi = nb - 1;   // largest row with items_before(row) <= q
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items_before<W, CW>(mid) <= q) lo = mid; else hi = mid - 1;
    }
    row = lo;
    chunk = (int)(q - items_before<W, CW>(lo));
}

struct ChainBars {
    uint64_t bfull[NBUF], bempty[NBUF], xfull[XR], xempty[XR];
    uint64_t tfull[2];    // band tiles of a step landed (bulk path), by step parity
    int abort;
};

// the s-th step (s >= 1) stages its band tiles into buffer s & 1: the phase of
// tfull[s & 1] it completes
LNB_DEV uint32_t tile_phase(int s) { return (uint32_t)(((s & 1) ? (s - 1) >> 1 : (s - 2) >> 1) & 1); }
static_assert(Cfg<float>::W * 64 <= NCOMP && Cfg<double>::W * 64 <= NCOMP, "one tile column per compute thread");

// wait for copies this CTA issued before it leaves: bounded by budget_ns, and
// unlike mbar_wait not cut short by an abort or a recorded timeout
LNB_DEV void drain_wait(uint64_t *bar, uint32_t parity, long long budget_ns)
{
    const uint64_t t0 = globaltimer();
    while (!tc::mbar_try_wait(bar, parity))
        if ((long long)(globaltimer() - t0) > budget_ns) return;
}

template <typename TT, int NR, bool TR>
__global__ void __launch_bounds__(NTHR, 1) k_trsm_chain(Args<TT> a, const __grid_constant__ CUtensorMap tmT)
{
    constexpr int W = Cfg<TT>::W, CW = Cfg<TT>::CW;
    constexpr int LD = Ld<TT, TR>::v;
    constexpr int TS = TH * LD;           // elements per staged tile
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ int64_t s_item;
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    const int nb = a.nb;

    if (tid == 0) s_item = atomicAdd(a.ticket, 1);
    __syncthreads();
    int64_t item = s_item;

    if (item == 0) {
        // ================= the chain CTA =================
        // tiles 1024-byte aligned (the swizzled TMA layout needs it)
        unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
        TT *tiles = reinterpret_cast<TT *>(sm);                                       // [2][W][TS]
        double *ring = reinterpret_cast<double *>(sm + sizeof(TT) * 2 * W * TS);       // [W+1][NR][64]
        double *bbuf = ring + (W + 1) * NR * TH;                                      // [NBUF][NR][64]
        double *accs = bbuf + NBUF * NR * TH;                                         // [NR][64]
        ChainBars *cb = reinterpret_cast<ChainBars *>(accs + NR * TH);
        if (tid == 0) {
            for (int q = 0; q < NBUF; ++q) { tc::mbar_init(&cb->bfull[q], 8); tc::mbar_init(&cb->bempty[q], NCOMP); }
            for (int q = 0; q < XR; ++q) { tc::mbar_init(&cb->xfull[q], NCOMP); tc::mbar_init(&cb->xempty[q], 1); }
            tc::mbar_init(&cb->tfull[0], 1);
            tc::mbar_init(&cb->tfull[1], 1);
            cb->abort = 0;
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        const int warp = tid >> 5, lane = tid & 31;

        if (warp == 8) {
            // ---- publisher: X_p visible GPU-wide, then ready[p].  One fence covers
            //      every block the compute warps have finished by then. ----
            if (lane == 0) {
                int p = 0;
                while (p < nb) {
                    if (!tc::mbar_wait(&cb->xfull[p % XR], (p / XR) & 1, a.wait_ns, &cb->abort, a.st)) {
                        cb->abort = 1;
                        atomicCAS(&a.st->timeout, 0, 4);
                        a.st->timeout_item = p;
                        break;
                    }
                    int q = p + 1;
                    while (q < nb && q < p + XR && tc::mbar_try_wait(&cb->xfull[q % XR], (q / XR) & 1)) ++q;
                    fence_acq_rel_gpu();
                    for (int t = p; t < q; ++t) {
                        st_relaxed(&a.ready[t], 1);
                        tc::mbar_arrive(&cb->xempty[t % XR]);
                    }
                    p = q;
                }
            }
            return;
        }
        if (warp == 9) {
            // ---- loader: 4 groups of 8 lanes; group g stages the B rows of chain
            //      positions p = g (mod 4) into slot g once the row's items are done.
            //      16-byte copies from L2 land asynchronously and complete the slot's
            //      mbarrier, so a group polls its next row while copies are in flight. ----
            const int g = lane >> 3, gl = lane & 7;
            const unsigned gmask = 0xffu << (8 * g);
            const bool vecB = ((uintptr_t)a.B % 16 == 0) && (a.ldb % 2 == 0);
            for (int p = g; p < nb; p += NBUF) {
                bool ok = true;
                if (gl == 0) {
                    if (p >= NBUF)
                        ok = tc::mbar_wait(&cb->bempty[g], ((p / NBUF) - 1) & 1, a.wait_ns, &cb->abort, a.st);
                    if (ok) ok = wait_geq(&a.cnt[p], need_of<W, CW>(p), a.wait_ns, a.st);
                }
                ok = __shfl_sync(gmask, ok, 8 * g);
                if (!ok) {
                    if (gl == 0) { cb->abort = 1; atomicCAS(&a.st->timeout, 0, 5); a.st->timeout_item = p; }
                    break;
                }
                const int i = blk(a, p);
                const int64_t oi = (int64_t)i * TH;
                const int in_ = blen(a, i);
                double *dst = bbuf + g * NR * TH;
                if (vecB) {
#pragma unroll
                    for (int q = 0; q < 4 * NR; ++q) {
                        const int pr = gl + 8 * q, r = pr / 32, mm = 2 * (pr % 32);
                        const int nv = (r < a.nrhs) ? max(0, min(2, in_ - mm)) : 0;
                        cp_async16_n(dst + r * TH + mm, nv ? a.B + (oi + mm) + (int64_t)r * a.ldb : a.B, 8 * nv);
                    }
                    cp_async_mbar_arrive(&cb->bfull[g]);
                } else {
#pragma unroll
                    for (int q = 0; q < 8 * NR; ++q) {
                        const int idx = gl + 8 * q, r = idx / TH, mm = idx % TH;
                        dst[idx] = (mm < in_ && r < a.nrhs) ? __ldcg(a.B + (oi + mm) + (int64_t)r * a.ldb) : 0.0;
                    }
                    __syncwarp(gmask);
                    tc::mbar_arrive(&cb->bfull[g]);
                }
            }
            cp_async_wait<0>();
            return;
        }

        // ---- compute warps ----
        const int m = tid >> 2, kq = tid & 3;
        TT dA[16], dB[16];
        load_dinv<TR, TT>(a.dinv, blk(a, 0), m, kq, dA);
        bool okp = true;
        // Whole 64 x 64 tiles with 16-byte-aligned columns: one bulk copy per
        // tile column (one per compute thread), counted on tfull; otherwise
        // cp.async in 16-byte pieces.
        const bool bulk = a.vec && (a.n % TH == 0);
        int staged = 0, consumed = 0;   // last step whose band tiles were issued / have landed (bulk path)
        // one chain step at position p; dcur holds inv(op T_pp), dnext receives the next one
        auto step = [&](int p, TT (&dcur)[16], TT (&dnext)[16]) -> bool {
            bool okt = true;
            if (!bulk) cp_async_wait<0>();
            else if (p >= 1) {
                okt = tc::mbar_wait(&cb->tfull[p & 1], tile_phase(p), a.wait_ns, &cb->abort, a.st);
                if (okt) consumed = p;
            }
            if (!bar_and(1, NCOMP, okt && okp && !*(volatile int *)&cb->abort)) return false;
            // prefetch the band tiles of position p+1 and its inverse
            if (p + 1 < nb) {
                const int ip = blk(a, p + 1);
                TT *tb = tiles + ((p + 1) & 1) * W * TS;
                if (a.tma) {
                    // one thread: two 32-row boxes per band tile, counted on tfull
                    if (tid == 0) {
                        const int ntl = p + 1 < W ? p + 1 : W;
                        tc::mbar_arrive_expect_tx(&cb->tfull[(p + 1) & 1], ntl * TH * TH * (int)sizeof(TT));
                        for (int k = 1; k <= ntl; ++k) {
                            const int jb = blk(a, p + 1 - k);
                            const int rb = TR ? jb : ip, cbk = TR ? ip : jb;
#pragma unroll
                            for (int h = 0; h < 2; ++h)
                                tc::tma_load_2d(tb + (k - 1) * TS + h * 2048, &tmT, &cb->tfull[(p + 1) & 1],
                                                rb * TH + 32 * h, cbk * TH);
                        }
                    }
                    staged = p + 1;
                } else if (bulk) {
                    const int ntl = p + 1 < W ? p + 1 : W;
                    if (tid == 0) tc::mbar_arrive_expect_tx(&cb->tfull[(p + 1) & 1], ntl * TH * TH * (int)sizeof(TT));
                    const int k = 1 + (tid >> 6), col = tid & 63;
                    if (k <= ntl) {
                        const int jb = blk(a, p + 1 - k);
                        const int rb = TR ? jb : ip, cbk = TR ? ip : jb;
                        bulk_copy_g2s(tb + (k - 1) * TS + col * LD,
                                      a.T + (int64_t)rb * TH + ((int64_t)cbk * TH + col) * a.ldt,
                                      TH * (uint32_t)sizeof(TT), &cb->tfull[(p + 1) & 1]);
                    }
                    staged = p + 1;
                } else {
#pragma unroll
                    for (int k = 1; k <= W; ++k)
                        if (p + 1 - k >= 0)
                            stage_tile<TT, TR>(a, tb + (k - 1) * TS, ip, blk(a, p + 1 - k), tid, NCOMP);
                }
                load_dinv<TR, TT>(a.dinv, ip, m, kq, dnext);
            }
            if (!bulk) cp_async_commit();
            // L2 prefetch PF steps ahead (band tiles, one column per thread, and the
            // diagonal inverse), so the cp.async of the next step is served from L2
            if (a.tma) {
                if (tid == 0 && p + PF < nb) {
                    const int ip = blk(a, p + PF);
                    for (int k = 1; k <= W && p + PF - k >= 0; ++k) {
                        const int jb = blk(a, p + PF - k);
                        const int rb = TR ? jb : ip, cbk = TR ? ip : jb;
                        prefetch_box_l2(&tmT, rb * TH, cbk * TH);
                        prefetch_box_l2(&tmT, rb * TH + 32, cbk * TH);
                    }
                    prefetch_l2(a.dinv + (int64_t)ip * TH * TH, TH * TH * sizeof(TT));
                }
            } else if (a.vec && p + PF < nb) {
                const int k = 1 + (tid >> 6);
                if (k <= W && p + PF - k >= 0)
                    prefetch_tile_col<TT, TR>(a, blk(a, p + PF), blk(a, p + PF - k), tid & 63);
                if (tid == 255) prefetch_l2(a.dinv + (int64_t)blk(a, p + PF) * TH * TH, TH * TH * sizeof(TT));
            }
            // band: sum_k op(T)(i, i-k) X_{p-k}
            double part[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) part[r] = 0.0;
#pragma unroll
            for (int k = 1; k <= W; ++k)
                if (p - k >= 0) {
                    const TT *tk = tiles + (p & 1) * W * TS + (k - 1) * TS;
                    const double *xk = ring + ((p - k) % (W + 1)) * NR * TH;
                    if constexpr (sizeof(TT) == 4) {
                        if (a.tma) gemv_tile_sw<NR, TR>(reinterpret_cast<const float *>(tk), xk, m, kq, part);
                        else gemv_tile<TT, NR, TR>(tk, xk, m, kq, part);
                    } else {
                        gemv_tile<TT, NR, TR>(tk, xk, m, kq, part);
                    }
                }
            quad_sum<NR>(part);
            const int slot = p % NBUF;
            const bool okb = tc::mbar_wait(&cb->bfull[slot], (p / NBUF) & 1, a.wait_ns, &cb->abort, a.st);
            if (okb) {
                const double *bs = bbuf + slot * NR * TH;
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if ((r & 3) == kq) accs[r * TH + m] = bs[r * TH + m] - part[r];
            }
            tc::mbar_arrive(&cb->bempty[slot]);
            if (!bar_and(1, NCOMP, okb)) return false;
            // X_p = inv(op T_pp) acc
            double xs[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) xs[r] = 0.0;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int k = kd<TR>(kq, j);
#pragma unroll
                for (int r = 0; r < NR; ++r) xs[r] = fma((double)dcur[j], accs[r * TH + k], xs[r]);
            }
            quad_sum<NR>(xs);
            const int i = blk(a, p);
            const int64_t oi = (int64_t)i * TH;
            const int in_ = blen(a, i);
            double *xr = ring + (p % (W + 1)) * NR * TH;
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if ((r & 3) == kq) {
                    xr[r * TH + m] = xs[r];
                    if (m < in_ && r < a.nrhs) a.B[(oi + m) + (int64_t)r * a.ldb] = xs[r];
                }
            okp = true;
            if (p >= XR) okp = tc::mbar_wait(&cb->xempty[p % XR], ((p / XR) - 1) & 1, a.wait_ns, &cb->abort, a.st);
            tc::mbar_arrive(&cb->xfull[p % XR]);
            return true;
        };
        for (int p = 0; p < nb; p += 2) {
            bool ok = step(p, dA, dB);
            if (ok && p + 1 < nb) ok = step(p + 1, dB, dA);
            if (!ok) {
                cp_async_wait<0>();
                // bulk copies still in flight land before the CTA leaves (bounded)
                if (bulk && staged > consumed) drain_wait(&cb->tfull[staged & 1], tile_phase(staged), a.wait_ns);
                if (tid == 0) { cb->abort = 1; atomicCAS(&a.st->timeout, 0, 3); a.st->timeout_item = p; }
                return;
            }
        }
        cp_async_wait<0>();
        return;
    }

    // ================= worker CTAs =================
    // tiles 1024-byte aligned (the swizzled TMA layout needs it)
    unsigned char *wsm = reinterpret_cast<unsigned char *>(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
    TT *wbuf = reinterpret_cast<TT *>(wsm);                                        // [2][CW][TS]
    double *xw = reinterpret_cast<double *>(wsm + sizeof(TT) * 2 * CW * TS);       // [CW][NR][64]
    uint64_t *wfull = reinterpret_cast<uint64_t *>(xw + CW * NR * TH);             // [2], TMA staging
    const int64_t total = 1 + items_before<W, CW>(nb);
    const int m = tid >> 2, kq = tid & 3;
    int buf = 0;
    int row = 0, chunk = 0;
    // TMA staging: thread 0 issues two 32-row boxes per tile, counted on wfull[b];
    // use[b] counts the completed phases of wfull[b], pend[b] marks boxes in flight
    int use[2] = {0, 0}, pend[2] = {0, 0};
    if (a.tma) {
        if (tid == 0) {
            tc::mbar_init(&wfull[0], 1);
            tc::mbar_init(&wfull[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    auto stage_item = [&](int b, int irow, int j0, int j1) {
        if (a.tma) {
            if (tid == 0) {
                tc::mbar_arrive_expect_tx(&wfull[b], (j1 - j0) * TH * TH * (int)sizeof(TT));
                for (int jj = j0; jj < j1; ++jj) {
                    const int i = blk(a, irow), j = blk(a, jj);
                    const int rb = TR ? j : i, cbk = TR ? i : j;
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        tc::tma_load_2d(wbuf + b * CW * TS + (jj - j0) * TS + h * 2048, &tmT, &wfull[b],
                                        rb * TH + 32 * h, cbk * TH);
                }
            }
            pend[b] = 1;
        } else {
            for (int jj = j0; jj < j1; ++jj)
                stage_tile<TT, TR>(a, wbuf + b * CW * TS + (jj - j0) * TS, blk(a, irow), blk(a, jj), tid, NTHR);
        }
    };
    // boxes in flight land before the CTA leaves (bounded)
    auto drain = [&]() {
        for (int b = 0; b < 2; ++b)
            if (pend[b]) drain_wait(&wfull[b], (uint32_t)(use[b] & 1), a.wait_ns);
    };
    if (item < total) {
        decode<W, CW>(item - 1, nb, row, chunk);
        const int j0 = chunk * CW, j1 = min(j0 + CW, row - W);
        stage_item(0, row, j0, j1);
    }
    cp_async_commit();
    while (item < total) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int64_t next = s_item;
        int nrow = 0, nchunk = 0;
        if (next < total) {
            decode<W, CW>(next - 1, nb, nrow, nchunk);
            const int j0 = nchunk * CW, j1 = min(j0 + CW, nrow - W);
            stage_item(buf ^ 1, nrow, j0, j1);
        }
        cp_async_commit();
        const int j0 = chunk * CW, j1 = min(j0 + CW, row - W);
        if (tid == 0) {
            s_ok = wait_geq(&a.ready[j1 - 1], 1, a.wait_ns, a.st);
            if (!s_ok) { atomicCAS(&a.st->timeout, 0, 6); a.st->timeout_item = (int)item; }
        }
        __syncthreads();
        if (!s_ok) { cp_async_wait<0>(); drain(); return; }
        for (int idx = tid; idx < (j1 - j0) * NR * TH; idx += NTHR) {
            const int t = idx / (NR * TH), r = (idx / TH) % NR, k = idx % TH;
            const int j = blk(a, j0 + t);
            const int64_t oj = (int64_t)j * TH;
            xw[idx] = (k < blen(a, j) && r < a.nrhs) ? __ldcg(a.B + (oj + k) + (int64_t)r * a.ldb) : 0.0;
        }
        if (a.tma) {
            volatile int no_abort = 0;
            const bool okw = tc::mbar_wait(&wfull[buf], (uint32_t)(use[buf] & 1), a.wait_ns, &no_abort, a.st);
            if (okw) { ++use[buf]; pend[buf] = 0; }
            if (!__syncthreads_and(okw)) {
                if (tid == 0) { atomicCAS(&a.st->timeout, 0, 7); a.st->timeout_item = (int)item; }
                drain();
                return;
            }
        } else {
            cp_async_wait<1>();
            __syncthreads();
        }
        if (tid < NCOMP) {
            double part[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) part[r] = 0.0;
            for (int jj = j0; jj < j1; ++jj) {
                const TT *tk = wbuf + buf * CW * TS + (jj - j0) * TS;
                const double *xk = xw + (jj - j0) * NR * TH;
                if constexpr (sizeof(TT) == 4) {
                    if (a.tma) gemv_tile_sw<NR, TR>(reinterpret_cast<const float *>(tk), xk, m, kq, part);
                    else gemv_tile<TT, NR, TR>(tk, xk, m, kq, part);
                } else {
                    gemv_tile<TT, NR, TR>(tk, xk, m, kq, part);
                }
            }
            quad_sum<NR>(part);
            const int i = blk(a, row);
            const int64_t oi = (int64_t)i * TH;
            const int in_ = blen(a, i);
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if ((r & 3) == kq && m < in_ && r < a.nrhs)
                    atomicAdd(a.B + (oi + m) + (int64_t)r * a.ldb, -part[r]);
        }
        // the CTA barrier orders every thread's updates before thread 0's
        // GPU-scope release fence, which publishes them with the counter
        __syncthreads();
        if (tid == 0) {
            fence_acq_rel_gpu();
            atomicAdd(&a.cnt[row], 1);
        }
        item = next; row = nrow; chunk = nchunk; buf ^= 1;
    }
    cp_async_wait<0>();
}

template <typename TT, int NR, bool TR>
constexpr size_t smem_bytes()
{
    constexpr int W = Cfg<TT>::W, CW = Cfg<TT>::CW;
    constexpr size_t TSB = sizeof(TT) * TH * Ld<TT, TR>::v;
    constexpr size_t chainb =
        1024 + 2 * W * TSB + sizeof(double) * ((W + 1) + NBUF + 1) * NR * TH + sizeof(ChainBars);
    constexpr size_t workb = 1024 + 2 * CW * TSB + sizeof(double) * CW * NR * TH + 16;
    return chainb > workb ? chainb : workb;
}

template <typename TT, int NR, bool TR>
int launch(const Args<TT> &a, const CUtensorMap &tm, lnb_stream_t s)
{
    constexpr int W = Cfg<TT>::W, CW = Cfg<TT>::CW;
    constexpr size_t smem = smem_bytes<TT, NR, TR>();
    static_assert(smem <= 227 * 1024, "chain solve shared memory");
    cudaError_t e = cudaFuncSetAttribute(k_trsm_chain<TT, NR, TR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return (int)e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // worker items: G(nb - 1 - W)
    int64_t S = (int64_t)a.nb - 1 - W, witems = 0;
    if (S > 0) witems = CW * (S / CW) * (S / CW + 1) / 2 + (S % CW) * (S / CW + 1);
    int64_t grid = 1 + witems;
    if (grid > sms) grid = sms;
    k_trsm_chain<TT, NR, TR><<<(unsigned)grid, NTHR, smem, s>>>(a, tm);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}

// FP32 n x n column-major T (ld ldt) as a 2D tensor map with 32 x 64 boxes in
// the 128-byte-swizzled layout; 0 on success
typedef CUresult (*EncodeTiledFnC)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static int tile_map(CUtensorMap *m, const void *T, int64_t n, int64_t ldt)
{
    static EncodeTiledFnC fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return -1;
        fn = (EncodeTiledFnC)p;
    }
    cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)ldt * 4};
    cuuint32_t box[2] = {32, 64};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(T), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : -1;
}

template <typename TT>
int trsm_chain(char uplo, char trans, int64_t n, int64_t nrhs, const TT *T, int64_t ldt, const TT *dinv,
               double *B, int64_t ldb, int *sync, lnb_status_t *st, long long wait_ns, lnb_stream_t s)
{
    Args<TT> a;
    a.T = T; a.ldt = ldt; a.dinv = dinv; a.B = B; a.ldb = ldb; a.n = n; a.nrhs = (int)nrhs;
    a.nb = (int)((n + TH - 1) / TH);
    const bool lowerop = (uplo == 'L') == (trans == 'N');
    a.fwd = lowerop ? 1 : 0;
    a.vec = ((uintptr_t)T % 16 == 0) && ((ldt * (int64_t)sizeof(TT)) % 16 == 0);
    a.ticket = sync; a.cnt = sync + 4; a.ready = sync + 4 + a.nb;
    a.st = st; a.wait_ns = wait_ns;
    // FP32 T in whole 64-blocks with 16-byte-aligned columns: the chain CTA's
    // band tiles come through a tensor map (boxes 32 rows x 64 columns, 128-byte swizzle)
    CUtensorMap tm;
    memset(&tm, 0, sizeof tm);
    a.tma = 0;
    const char *env = getenv("LNB_CHAIN_TMA");   /* 0: stage by bulk copies instead */
    const bool want = !(env && *env && atoi(env) == 0);
    if (want && sizeof(TT) == 4 && a.vec && n % TH == 0 && tile_map(&tm, T, n, ldt) == 0) a.tma = 1;
    const bool tr = trans == 'T';
    if (nrhs <= 1) return tr ? launch<TT, 1, true>(a, tm, s) : launch<TT, 1, false>(a, tm, s);
    if (nrhs <= 2) return tr ? launch<TT, 2, true>(a, tm, s) : launch<TT, 2, false>(a, tm, s);
    if (nrhs <= 4) return tr ? launch<TT, 4, true>(a, tm, s) : launch<TT, 4, false>(a, tm, s);
    return tr ? launch<TT, 8, true>(a, tm, s) : launch<TT, 8, false>(a, tm, s);
}

}  // namespace chain
}  // namespace lnb

// sync must hold lnb_trsm_sync_ints(n, 64) zeroed ints (ticket first).
extern "C" int lnb_k_trsm_chain_f64(char uplo, char trans, int64_t n, int64_t nrhs, const double *T, int64_t ldt,
                                    const double *dinv, double *B, int64_t ldb, int *sync, lnb_status_t *st,
                                    long long wait_ns, lnb_stream_t s)
{
    if (nrhs > 8) return (int)cudaErrorInvalidValue;
    return lnb::chain::trsm_chain<double>(uplo, trans, n, nrhs, T, ldt, dinv, B, ldb, sync, st, wait_ns, s);
}
extern "C" int lnb_k_trsm_chain_f32(char uplo, char trans, int64_t n, int64_t nrhs, const float *T, int64_t ldt,
                                    const float *dinv, double *B, int64_t ldb, int *sync, lnb_status_t *st,
                                    long long wait_ns, lnb_stream_t s)
{
    if (nrhs > 8) return (int)cudaErrorInvalidValue;
    return lnb::chain::trsm_chain<float>(uplo, trans, n, nrhs, T, ldt, dinv, B, ldb, sync, st, wait_ns, s);
}
