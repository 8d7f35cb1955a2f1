// mpmw_tma.cuh -- Tensor Memory Accelerator (TMA) tile loads for sm_100a.
//
// Device side: an mbarrier in shared memory, one elected thread issues
// cp.async.bulk.tensor.4d (no multicast) with complete_tx accounting, every
// thread waits on the barrier's phase for a bounded time.
// Host side: CUtensorMap descriptors of grid velocity arrays, cached per
// (pointer, dims).
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace mpmw {

constexpr int kTileEdge = 8;                                       // nodes per tile edge
constexpr int kTileNodes = kTileEdge * kTileEdge * kTileEdge;      // 512
constexpr unsigned kTileBytes = kTileNodes * 16u;                  // float4 per node
constexpr int kMbarMaxPolls = 1 << 24;  // also bounded by kMbarWaitNs

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// invalidate before the barrier's shared memory is used again (another
// mbarrier.init included)
__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, unsigned phase)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Potentially blocking test: the hardware suspends the thread until the phase
// completes or about `hint_ns` nanoseconds pass, whichever is first.
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase, unsigned hint_ns)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Wait for phase `phase` of the barrier for at most kMbarWaitNs of wall time;
// false if it never completed.  Each poll suspends the warp in hardware (at
// most kMbarSuspendNs), so a warp waiting on a copy does not take issue slots
// from the warps that compute; the wall-time bound is checked between polls.
constexpr uint64_t kMbarWaitNs = 200ull * 1000ull * 1000ull;  // 200 ms
constexpr unsigned kMbarSuspendNs = 20000u;                   // 20 us per poll at most
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned phase)
{
    if (mbar_test_wait(bar, phase)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (int i = 0; i < kMbarMaxPolls; ++i) {
        if (mbar_try_wait(bar, phase, kMbarSuspendNs)) return true;
        if (globaltimer_ns() - t0 > kMbarWaitNs) return false;
    }
    return false;
}

// 4-D tiled tensor load (coordinates innermost first) into shared memory,
// completion signalled on `bar`.  c0 must be a multiple of 16 bytes / element
// size (it is 0 for the float4 node records loaded here).
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completion signalled on `bar`.
// dst and src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Host: tensor map over a (nx, ny, nz, 4) float32 grid array, box
// (4, kTileEdge, kTileEdge, kTileEdge), zero fill outside the array.
// Returns false if the driver rejects the descriptor.
bool grid_tensor_map(const float *base, const int *dims, CUtensorMap *out);

}  // namespace mpmw
