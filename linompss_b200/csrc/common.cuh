// common.cuh -- device helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lnb_kern.h"

#define LNB_DEV __device__ __forceinline__

namespace lnb {

// ---- FP64 tensor-core MMA (DMMA), warp-synchronous ----------------------
// D(16x8) += A(16x4, row) * B(4x8, col).  Fragment ownership, g = lane>>2,
// t = lane&3:  a0 = A[g][t], a1 = A[g+8][t];  b0 = B[t][g];
// c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1].
LNB_DEV void dmma16x8x4(double (&c)[4], double a0, double a1, double b0)
{
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

// ---- cp.async (Ampere-style async copy global -> shared) ------------------
LNB_DEV uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 16-byte copy, zero-filled when !pred
LNB_DEV void cp_async16(void *smem, const void *gmem, bool pred)
{
    int n = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(n));
}
// 8-byte copy, zero-filled when !pred
LNB_DEV void cp_async8(void *smem, const void *gmem, bool pred)
{
    int n = pred ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(smem)),
                 "l"(gmem), "r"(n));
}
LNB_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
LNB_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---- bounded waits --------------------------------------------------------
LNB_DEV uint64_t globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
LNB_DEV int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
LNB_DEV void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Spin until *flag >= target; returns false if wait_ns of device time passed
// first or another waiter already reported a timeout.
LNB_DEV bool wait_geq(const int *flag, int target, long long wait_ns, const lnb_status_t *st)
{
    if (ld_acquire(flag) >= target) return true;
    uint64_t t0 = globaltimer();
    unsigned ns = 32;
    while (true) {
        if (ld_acquire(flag) >= target) return true;
        if (ld_acquire(&st->timeout) != 0) return false;
        if ((long long)(globaltimer() - t0) > wait_ns) return false;
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;   // short cap: these waits sit on dependency chains
    }
}

}  // namespace lnb
