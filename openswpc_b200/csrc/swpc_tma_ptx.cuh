// swpc_tma_ptx.cuh -- the mbarrier and bulk-tensor-copy primitives of the
// TMA-staged kernels (swpc3d_tma.cu, swpc2d_tma.cu), as inline PTX for
// sm_100a.  No multicast: every copy lands in the issuing CTA's own shared
// memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace swpc {
namespace tma {

constexpr unsigned long long kWaitNs = 100000000ull;   // 100 ms: a tile copy takes microseconds

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// tiled tensor copies global -> shared, completion counted on bar
__device__ __forceinline__ void load_3d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                        uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// first 128-byte aligned address of the dynamic shared memory (TMA
// destinations); the launches reserve 128 bytes for the shift
__device__ __forceinline__ float *aligned128(unsigned char *p) {
    const unsigned a = smem_u32(p);
    return reinterpret_cast<float *>(p + ((128u - (a & 127u)) & 127u));
}

__device__ __forceinline__ unsigned long long gtime() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Barrier set-up by the lead thread, before it issues the tile copies.  The
// other threads touch the barrier only after the block synchronises.
__device__ __forceinline__ void stage_init(uint64_t *bar, unsigned bytes) {
    mbar_init(bar, 1);
    fence_barrier_init();
    mbar_expect_tx(bar, bytes);
}

// Wait limit of a CTA, read by the lead thread after it issued its copies
// (the read travels with them): kWaitNs, or kWaitAfterErrNs once an earlier
// tile copy of the launch did not complete, so that a launch whose copies
// fail ends quickly.
constexpr unsigned long long kWaitAfterErrNs = 1000000ull;   // 1 ms
__device__ __forceinline__ unsigned long long wait_limit(const int *err) {
    return *reinterpret_cast<const volatile int *>(err) == 0 ? kWaitNs : kWaitAfterErrNs;
}

// Bounded wait for the tile copies.  After `limit` ns the kernel raises the
// error word, waits once more (bounded) for its copies in flight, and the
// caller skips the staged cells.
__device__ __forceinline__ bool wait_tiles(uint64_t *bar, int *err, unsigned long long limit) {
    const unsigned long long t0 = gtime();
    while (!mbar_try_wait(bar, 0)) {
        if (gtime() - t0 > limit) {
            atomicExch(err, 1);
            const unsigned long long t1 = gtime();
            while (!mbar_try_wait(bar, 0) && gtime() - t1 < limit) {
            }
            return false;
        }
    }
    return true;
}

__host__ __device__ constexpr int up32(int n) { return (n + 31) / 32 * 32; }

}  // namespace tma
}  // namespace swpc
