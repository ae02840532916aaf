// k_chol_dag.cu -- FP64 tile Cholesky as ONE persistent launch that walks the
// task DAG on the device.
//
// Reference: dchol_rl (chol_rlmain.c:22-53) issues POTRF / TRSM / SYRK / GEMM
// tile tasks that the OmpSs runtime orders by their data dependencies (keyed
// on tile base addresses, tasks_potrf.h:19) and by priority (POTRF and TRSM
// at 9999 over GEMM and SYRK at 9, chol_rlmain.c:14-19).  Here the DAG lives
// on the GPU:
//
//   * The factor is cut into 64 x 64 tiles (the last row and column ragged).
//     A task produces one finished tile L_ij (i >= j):
//         S    = A_ij - sum_{k<j} L_ik L_jk^T          (SYRK for i == j, GEMMs otherwise)
//         i==j : L_jj = potrf(S), W_j = L_jj^-1       (POTRF, and the inverse for the tiles below)
//         i> j : L_ij = S W_j^T                       (TRSM as a product with the inverse)
//     The sum runs left-looking in 32-column chunks on DMMA (mma.sync
//     m16n8k4 f64), each chunk staged by cp.async once the two tiles it reads
//     are final.
//   * Tasks are handed out by an atomic ticket in column order, the diagonal
//     task first in each column: the device form of the reference's priorities
//     (the critical POTRF/TRSM chain of column j goes out before any work of
//     column j+1).  A task waits only on tiles of earlier columns and on the
//     diagonal tile of its own column, all with smaller tickets, which running
//     CTAs hold; so the walk cannot deadlock whatever the residency.
//   * Every tile has a done flag (release by one thread after a CTA barrier,
//     acquire by one thread before a CTA barrier).  Every wait is bounded by
//     wait_ns of device time; a wait that runs out sets st->timeout and the
//     CTA drains its copies and stops, and the other waiters see the timeout
//     and stop too.
//   * A non-positive pivot is reported LAPACK-style in st->info (1-based
//     global column); the columns before it are final for every row, and the
//     walk still finishes every task (with the inverse's rows past the failure
//     replaced by identity rows), so nothing waits forever.
#include "common.cuh"

namespace lnb {
namespace dag {

constexpr int TS = 64;              // tile order
constexpr int NT = 128;             // threads per CTA (4 warps, 2 x 2 warp grid of 32 x 32)
constexpr int BK = 32;              // K chunk
constexpr int LDK = TS + 4;         // k-major staged rows (= 4 mod 16 doubles: conflict-free fragments)
constexpr int CHUNK = BK * LDK;     // doubles per staged operand chunk
constexpr int LDS = TS + 1;         // row-major tile for the diagonal factor
constexpr int SMEM_STAGES = 2 * 2 * CHUNK * (int)sizeof(double);          // 2 stages x {A, B}
constexpr int SMEM_POTRF = (2 * TS * LDS + 32) * (int)sizeof(double);     // S, W and the pivot reciprocals
constexpr int SMEM = SMEM_STAGES > SMEM_POTRF ? SMEM_STAGES : SMEM_POTRF;

struct Args {
    double *A;
    int64_t lda, n;
    int nt, ntasks;
    double *W;              // nt inverses of the diagonal tiles, 64 x 64 column-major each
    int *done;              // done[k * nt + i]: tile (i, k) is final
    int *ticket;
    int ticket0;            // first ticket handed out (0; 1 only in the wait self-test)
    lnb_status_t *st;
    long long wait_ns;
};

// ---- one warp: Cholesky of a 32 x 32 block and its inverse ------------------
// S: row-major (ld lds), lower part read and written.  X: row-major (ld ldx),
// receives inv(L) (lower; zeros above).  rd: 32 doubles of scratch.
// Factor: lane r owns row r in registers; a runtime loop over the columns
// keeps a[0] the current column (the array shifts down by one per step, so
// every index is a compile-time constant) and reads L's finished column back
// from shared memory, where every lane reads the same word (a broadcast).
// Inverse: lane q forms column q of inv(L) by forward substitution with the
// stored reciprocal pivots, X[r][q] = (delta_rq - sum_{k<r} L[r][k] X[k][q]) / L[r][r].
// Returns the local column of the first non-positive pivot, or 32.  After a
// failure the failed pivot and the columns after it keep their updated values
// (LAPACK's potf2 stops there) and X's rows from the failure on are identity
// rows.
LNB_DEV int warp_potrf32_inv(double *S, int lds, double *X, int ldx, double *rd)
{
    const int lane = threadIdx.x & 31;
    double a[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) a[k] = (k <= lane) ? S[lane * lds + k] : 0.0;
    int fail = 32;
#pragma unroll 1
    for (int c = 0; c < 32; ++c) {
        const double d = __shfl_sync(0xffffffffu, a[0], c);
        if (!(d > 0.0)) {                                // warp-uniform: stop here
            fail = c;
#pragma unroll
            for (int k = 0; k < 32; ++k)
                if (c + k <= lane) S[lane * lds + c + k] = a[k];
            break;
        }
        const double rs = rsqrt(d);
        if (lane >= c) S[lane * lds + c] = (lane == c) ? d * rs : a[0] * rs;
        if (lane == c) rd[c] = rs;
        const double l = a[0] * rs;
        __syncwarp();
#pragma unroll
        for (int k = 1; k < 32; ++k) {
            const double lk = S[((c + k) & 31) * lds + c];
            if (c + k <= lane) a[k] = fma(-l, lk, a[k]);
        }
#pragma unroll
        for (int k = 0; k < 31; ++k) a[k] = a[k + 1];
        a[31] = 0.0;
    }
    __syncwarp();
    double x[32];
#pragma unroll
    for (int r = 0; r < 32; ++r) {
        double sum = (r == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int k = 0; k < r; ++k) sum = fma(-S[r * lds + k], x[k], sum);
        x[r] = (r < fail) ? sum * rd[r < fail ? r : 0] : ((r == lane) ? 1.0 : 0.0);
    }
#pragma unroll
    for (int r = 0; r < 32; ++r) X[r * ldx + lane] = (r >= lane) ? x[r] : 0.0;
    __syncwarp();
    return fail;
}

// ---- the CTA: factor and invert the 64 x 64 tile S (row-major, ld LDS) -------
// 2 x 2 blocks of 32:  L00 = potrf(S00);  L10 = S10 W00^T;  S11 -= L10 L10^T;
// L11 = potrf(S11);  W10 = -W11 (L10 W00).  W (row-major, ld LDS) receives
// inv(L).  Returns the first failed local column, or 64.
LNB_DEV int cta_potrf64_inv(double *S, double *W, int *s_fail, double *rd)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int idx = tid; idx < 32 * 32; idx += NT) W[(idx >> 5) * LDS + 32 + (idx & 31)] = 0.0;
    if (warp == 0) {
        const int f = warp_potrf32_inv(S, LDS, W, LDS, rd);
        if (lane == 0) s_fail[0] = f;
    }
    __syncthreads();
    const int f0 = s_fail[0];
    // L10[r][c] = sum_{p <= c} S10[r][p] W00[c][p]; thread: row 32 + lane, columns 8 warp .. + 8
    {
        const int r = 32 + lane, cb = 8 * warp;
        double o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = 0.0;
        for (int p = 0; p < 32; ++p) {
            const double s = S[r * LDS + p];
#pragma unroll
            for (int u = 0; u < 8; ++u) o[u] = fma(s, W[(cb + u) * LDS + p], o[u]);
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 8; ++u) S[r * LDS + cb + u] = o[u];
    }
    __syncthreads();
    if (f0 < 32) {
        // the trailing block is not factored: W11 = I, W10 = 0
        for (int idx = tid; idx < 32 * 64; idx += NT) {
            const int r = 32 + idx / 64, q = idx % 64;
            W[r * LDS + q] = (q == r) ? 1.0 : 0.0;
        }
        __syncthreads();
        return f0;
    }
    // S11 -= L10 L10^T on the lower part; thread: row 32 + lane, columns 32 + 8 warp .. + 8
    {
        const int r = 32 + lane, cb = 32 + 8 * warp;
        double o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = 0.0;
        for (int p = 0; p < 32; ++p) {
            const double s = S[r * LDS + p];
#pragma unroll
            for (int u = 0; u < 8; ++u) o[u] = fma(s, S[(cb + u) * LDS + p], o[u]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
            if (r >= cb + u) S[r * LDS + cb + u] -= o[u];
    }
    __syncthreads();
    if (warp == 0) {
        const int f = warp_potrf32_inv(S + 32 * LDS + 32, LDS, W + 32 * LDS + 32, LDS, rd);
        if (lane == 0) s_fail[1] = f;
    }
    __syncthreads();
    const int f1 = s_fail[1];
    // T = L10 W00 into the unused upper-right block of S: T[r][q] = sum_{p >= q} L10[r][p] W00[p][q]
    {
        const int r = lane, qb = 8 * warp;
        double o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = 0.0;
        for (int p = 0; p < 32; ++p) {
            const double l = S[(32 + r) * LDS + p];
#pragma unroll
            for (int u = 0; u < 8; ++u) o[u] = fma(l, W[p * LDS + qb + u], o[u]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) S[r * LDS + 32 + qb + u] = o[u];
    }
    __syncthreads();
    // W10[r][q] = -sum_{s <= r} W11[r][s] T[s][q]
    {
        const int r = lane, qb = 8 * warp;
        double o[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) o[u] = 0.0;
        for (int s = 0; s < 32; ++s) {
            const double w = W[(32 + r) * LDS + 32 + s];
#pragma unroll
            for (int u = 0; u < 8; ++u) o[u] = fma(w, S[s * LDS + 32 + qb + u], o[u]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) W[(32 + r) * LDS + qb + u] = -o[u];
    }
    __syncthreads();
    return f1 < 32 ? 32 + f1 : 64;
}

// ---- DMMA over one staged chunk: acc(64 x 64) += As^T Bs (k-major operands) ---
LNB_DEV void mma_chunk(double (&acc)[2][4][4], const double *as, const double *bs, int wm, int wn, int g, int t)
{
#pragma unroll
    for (int kq = 0; kq < BK / 4; ++kq) {
        const double *ak = as + (kq * 4 + t) * LDK + wm * 32;
        const double *bk = bs + (kq * 4 + t) * LDK + wn * 32;
        double a0[2], a1[2], b0[4];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi) {
            a0[mi] = ak[mi * 16 + g];
            a1[mi] = ak[mi * 16 + g + 8];
        }
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) b0[ni] = bk[ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) dmma16x8x4(acc[mi][ni], a0[mi], a1[mi], b0[ni]);
    }
}

// stage rows [r0, r0+64) x columns [c0, c0+32) of the column-major matrix as
// dst[kk][m] (k-major), rows at or past n zero-filled
LNB_DEV void stage_chunk(double *dst, const double *A, int64_t lda, int64_t n, int64_t r0, int64_t c0, bool vec,
                         int tid)
{
    if (vec) {
        for (int idx = tid; idx < BK * TS / 2; idx += NT) {
            const int kk = idx / (TS / 2), m2 = (idx % (TS / 2)) * 2;
            const int64_t r = r0 + m2;
            const double *g = A + r + (c0 + kk) * lda;
            if (r + 1 < n) {
                cp_async16(dst + kk * LDK + m2, g, true);
            } else {
                cp_async8(dst + kk * LDK + m2, r < n ? g : A, r < n);
                cp_async8(dst + kk * LDK + m2 + 1, A, false);
            }
        }
    } else {
        for (int idx = tid; idx < BK * TS; idx += NT) {
            const int kk = idx / TS, m = idx % TS;
            const int64_t r = r0 + m;
            cp_async8(dst + kk * LDK + m, r < n ? A + r + (c0 + kk) * lda : A, r < n);
        }
    }
}

// thread 0 waits for the flags, the CTA learns the outcome (false: give up)
LNB_DEV bool cta_wait(const int *f0, const int *f1, const Args &a, int site, int item, int *s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = wait_geq(f0, 1, a.wait_ns, a.st);
        if (ok && f1 != nullptr) ok = wait_geq(f1, 1, a.wait_ns, a.st);
        if (!ok && atomicCAS(&a.st->timeout, 0, site) == 0) a.st->timeout_item = item;
        *s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    return *s_ok != 0;
}

// fragment (mi, ni, q) of warp (wm, wn) -> tile row / column
LNB_DEV int frag_row(int wm, int mi, int g, int q) { return wm * 32 + mi * 16 + g + ((q & 2) ? 8 : 0); }
LNB_DEV int frag_col(int wn, int ni, int t, int q) { return wn * 32 + ni * 8 + 2 * t + (q & 1); }

// one task: produce tile (i, j); false if a wait gave up
LNB_DEV bool run_tile(const Args &a, int i, int j, double *sm, int *s_ok, int *s_fail)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1, g = lane >> 2, t = lane & 3;
    const int64_t r0 = (int64_t)i * TS, cj = (int64_t)j * TS;
    const int rows = (int)((a.n - r0) < TS ? (a.n - r0) : TS);       // valid rows of the tile
    const int cols = (int)((a.n - cj) < TS ? (a.n - cj) : TS);       // valid columns
    const bool vec = ((uintptr_t)a.A % 16 == 0) && (a.lda % 2 == 0);
    const int item = j * a.nt + i;

    // the tile's own entries, loaded early (used after the K loop)
    double acc[2][4][4], aij[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = frag_row(wm, mi, g, q), c = frag_col(wn, ni, t, q);
                acc[mi][ni][q] = 0.0;
                aij[mi][ni][q] = (r < rows && c < cols) ? __ldcg(a.A + (r0 + r) + (cj + c) * a.lda) : 0.0;
            }

    // ---- S = A_ij - sum_{k<j} L_ik L_jk^T, two stages of 32-column chunks ----
    // stage x: A operand at sm + 2 x CHUNK, B operand right after it
    auto As = [&](int x) { return sm + 2 * x * CHUNK; };
    auto Bs = [&](int x) { return sm + (2 * x + 1) * CHUNK; };
    const bool diag = (i == j);
    const int nch = 2 * j;
    const int *done_i = a.done + i, *done_j = a.done + j;     // + k * nt
    if (nch > 0) {
        if (!cta_wait(done_i, diag ? nullptr : done_j, a, 31, item, s_ok)) return false;
        stage_chunk(As(0), a.A, a.lda, a.n, r0, 0, vec, tid);
        if (!diag) stage_chunk(Bs(0), a.A, a.lda, a.n, cj, 0, vec, tid);
        cp_async_commit();
    }
    for (int c = 0; c < nch; ++c) {
        const int nc = c + 1;
        if (nc < nch) {
            if ((nc & 1) == 0) {
                const int k = nc >> 1;
                // chunk c's data may still be in flight: it stays counted in its group
                if (!cta_wait(done_i + (int64_t)k * a.nt, diag ? nullptr : done_j + (int64_t)k * a.nt, a, 32,
                              item, s_ok)) {
                    cp_async_wait<0>();
                    return false;
                }
            }
            stage_chunk(As(nc & 1), a.A, a.lda, a.n, r0, (int64_t)nc * BK, vec, tid);
            if (!diag) stage_chunk(Bs(nc & 1), a.A, a.lda, a.n, cj, (int64_t)nc * BK, vec, tid);
        }
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        mma_chunk(acc, As(c & 1), diag ? As(c & 1) : Bs(c & 1), wm, wn, g, t);
        __syncthreads();
    }
    cp_async_wait<0>();

    if (diag) {
        // ---- POTRF of the tile and its inverse ----
        double *S = sm, *W = sm + TS * LDS;
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = frag_row(wm, mi, g, q), c = frag_col(wn, ni, t, q);
                    // padding past the ragged edge factors as the identity
                    const double v = (r < rows && c < cols) ? aij[mi][ni][q] - acc[mi][ni][q] : (r == c ? 1.0 : 0.0);
                    S[r * LDS + c] = v;
                }
        __syncthreads();
        const int f = cta_potrf64_inv(S, W, s_fail, W + TS * LDS);
        if (tid == 0 && f < cols) atomicCAS(&a.st->info, 0, (int)(cj + f + 1));
        // L (lower part, valid rows/columns) and the inverse (whole 64 x 64, column-major)
        for (int idx = tid; idx < TS * TS; idx += NT) {
            const int c = idx / TS, r = idx % TS;
            if (r >= c && r < rows && c < cols) a.A[(cj + r) + (cj + c) * a.lda] = S[r * LDS + c];
            a.W[(int64_t)j * TS * TS + idx] = W[r * LDS + c];
        }
    } else {
        // ---- TRSM: L_ij = S W_j^T, S staged k-major as the A operand ----
        if (!cta_wait(a.done + (int64_t)j * a.nt + j, nullptr, a, 33, item, s_ok)) return false;
        const double *Wj = a.W + (int64_t)j * TS * TS;
        // W_j^T in two chunks of 32 rows p: B(p, q) = W[q][p] = Wj[q + 64 p], 64 contiguous doubles
        for (int h = 0; h < 2; ++h)
            for (int idx = tid; idx < BK * TS / 2; idx += NT) {
                const int kk = idx / (TS / 2), q2 = (idx % (TS / 2)) * 2;
                cp_async16(Bs(h) + kk * LDK + q2, Wj + q2 + (int64_t)(h * BK + kk) * TS, true);
            }
        cp_async_commit();
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = frag_row(wm, mi, g, q), c = frag_col(wn, ni, t, q);
                    As(c >> 5)[(c & 31) * LDK + r] = aij[mi][ni][q] - acc[mi][ni][q];
                    acc[mi][ni][q] = 0.0;
                }
        cp_async_wait<0>();
        __syncthreads();
        mma_chunk(acc, As(0), Bs(0), wm, wn, g, t);
        mma_chunk(acc, As(1), Bs(1), wm, wn, g, t);
#pragma unroll
        for (int mi = 0; mi < 2; ++mi)
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int r = frag_row(wm, mi, g, q), c = frag_col(wn, ni, t, q);
                    if (r < rows && c < cols) a.A[(r0 + r) + (cj + c) * a.lda] = acc[mi][ni][q];
                }
    }
    // publish: every thread's stores, then one GPU-scope release
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        st_release(a.done + (int64_t)j * a.nt + i, 1);
    }
    return true;
}

__global__ void __launch_bounds__(NT, 2) k_chol_dag_f64(Args a)
{
    extern __shared__ __align__(16) double sm[];
    __shared__ int s_task, s_ok, s_fail[2];
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_task = atomicAdd(a.ticket, 1) + a.ticket0;
        __syncthreads();
        const int tk = s_task;
        if (tk >= a.ntasks) break;
        // column j holds tickets [j nt - j (j-1)/2, + nt - j): diagonal first, then rows below
        int lo = 0, hi = a.nt - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            const int64_t start = (int64_t)mid * a.nt - (int64_t)mid * (mid - 1) / 2;
            if (start <= tk) lo = mid; else hi = mid - 1;
        }
        const int j = lo;
        const int i = j + (int)(tk - ((int64_t)j * a.nt - (int64_t)j * (j - 1) / 2));
        if (!run_tile(a, i, j, sm, &s_ok, s_fail)) break;
    }
}

}  // namespace dag
}  // namespace lnb

extern "C" int64_t lnb_chol_dag_ints(int64_t n)
{
    const int64_t nt = (n + lnb::dag::TS - 1) / lnb::dag::TS;
    return nt * nt + 32;
}
extern "C" int64_t lnb_chol_dag_w_doubles(int64_t n)
{
    const int64_t nt = (n + lnb::dag::TS - 1) / lnb::dag::TS;
    return nt * lnb::dag::TS * lnb::dag::TS;
}

// sync: lnb_chol_dag_ints(n) ints (zeroed here); W: lnb_chol_dag_w_doubles(n).
// ticket0: first task handed out (0; > 0 only in the wait self-test, where
// skipping the first diagonal tile leaves dependencies that nothing satisfies).
extern "C" int lnb_k_chol_dag_f64(double *A, int64_t lda, int64_t n, double *W, int *sync, lnb_status_t *st,
                                  long long wait_ns, int sms, int ticket0, lnb_stream_t s)
{
    using namespace lnb::dag;
    if (n <= 0) return 0;
    const int64_t nt = (n + TS - 1) / TS;
    if (nt > 8192) return (int)cudaErrorInvalidValue;
    Args a;
    a.A = A; a.lda = lda; a.n = n; a.nt = (int)nt; a.ntasks = (int)(nt * (nt + 1) / 2);
    a.W = W; a.ticket = sync; a.ticket0 = ticket0; a.done = sync + 32; a.st = st; a.wait_ns = wait_ns;
    cudaError_t e = cudaMemsetAsync(sync, 0, (size_t)lnb_chol_dag_ints(n) * sizeof(int), (cudaStream_t)s);
    if (e != cudaSuccess) return (int)e;
    e = cudaFuncSetAttribute(k_chol_dag_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    if (e != cudaSuccess) return (int)e;
    const int grid = (int)(a.ntasks < 2 * sms ? a.ntasks : 2 * sms);
    k_chol_dag_f64<<<grid, NT, SMEM, (cudaStream_t)s>>>(a);
    lnb_prof_count(1);
    return (int)cudaGetLastError();
}
