// mpmw_gridsync.cuh -- grid-wide barrier and dynamic tile tickets for the
// persistent (cooperative-launch) kernels: every CTA of such a grid is
// resident at once, so CTAs may wait for one another; every wait is bounded.
#pragma once
#include "mpmw_common.cuh"
#include "mpmw_tma.cuh"

namespace mpmw {

constexpr uint64_t kGridSyncWaitNs = 1000ull * 1000ull * 1000ull;  // 1 s per barrier at most
constexpr unsigned kGridSyncMaxPolls = 1u << 24;

// Grid-wide barrier on a monotonically increasing arrival counter (zeroed
// before the launch): each CTA adds one and waits until the count reaches the
// next multiple of gridDim.x.  The wait is bounded (kGridSyncWaitNs of
// %globaltimer and kGridSyncMaxPolls polls); a CTA that gives up reports
// MPMW_ST_TIMEOUT and the call returns false in all its threads, after which
// the kernel returns (the other CTAs then give up at their next barrier).
// Global memory written before the barrier by plain stores may be read after
// it by bulk or TMA copies (the async proxy): every thread orders its writes
// for that proxy before arriving, and the waiting thread again after the
// acquire, before any copy is issued.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ bool grid_sync(unsigned *arrive, uint32_t *status, int *s_ok)
{
    fence_proxy_async_global();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned old = atomicAdd(arrive, 1u);
        const unsigned target = (old / gridDim.x + 1u) * gridDim.x;
        int ok = 1;
        const uint64_t t0 = globaltimer_ns();
        unsigned polls = 0;
        for (;;) {
            unsigned now;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(now) : "l"(arrive) : "memory");
            if ((int)(now - target) >= 0) break;
            if (++polls > kGridSyncMaxPolls || globaltimer_ns() - t0 > kGridSyncWaitNs) {
                ok = 0;
                raise_status(status, MPMW_ST_TIMEOUT);
                break;
            }
            if (polls > 32) __nanosleep(64);
        }
        __threadfence();
        fence_proxy_async_global();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// The next tile of a dynamically scheduled phase for this CTA: one ticket
// per draw from a counter that only grows (modulo 2^32), `base` tickets drawn
// by earlier such phases (each phase draws its tiles plus one final ticket per
// CTA, fewer than 2^31 in all).
__device__ __forceinline__ int draw_tile(unsigned *tickets, unsigned base, int *s_tile)
{
    if (threadIdx.x == 0) *s_tile = (int)(atomicAdd(tickets, 1u) - base);
    __syncthreads();
    const int t = *s_tile;
    __syncthreads();
    return t;
}

}  // namespace mpmw
