// mpmw_common.cuh -- shared host/device plumbing of libmpmw.so
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <cuda_runtime.h>

#include "../../include/mpmw.h"

namespace mpmw {

constexpr int kBlock = 256;  // threads per CTA for particle and node kernels

// thread-local last error message (mpmw_last_error)
void set_error(const char *fmt, ...);

// returns MPMW_E_LAUNCH and records the message if the last launch failed
int check_launch(const char *what);

inline cudaStream_t as_stream(mpmw_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

#define MPMW_TRY_LAUNCH(what)                 \
    do {                                      \
        int _rc = ::mpmw::check_launch(what); \
        if (_rc != MPMW_OK) return _rc;       \
    } while (0)

// Particle indices, worklists and hash ids are 32-bit: an element count above
// 2^31 - 1 is an argument error.  Records the message and returns true then.
inline bool count_too_large(int64_t n, const char *what)
{
    if (n <= (int64_t)INT32_MAX) return false;
    set_error("%s: count %lld exceeds the maximum of %d", what, (long long)n, (int)INT32_MAX);
    return true;
}

inline unsigned grid_for(int64_t n, int block = kBlock)
{
    int64_t b = (n + block - 1) / block;
    return (unsigned)(b > 0 ? b : 1);
}

__device__ __forceinline__ void raise_status(uint32_t *status, uint32_t bits)
{
    if (status) atomicOr(status, bits);
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may begin while the kernel before it in the
// stream is still running; pdl_wait() blocks until that kernel has completed
// and its memory operations are visible, so it comes before any read of the
// predecessor's results.  pdl_trigger() lets the next such kernel's CTAs be
// scheduled once every CTA of this grid has issued it (they then wait in
// their own pdl_wait).  Both are no-ops in a kernel launched the usual way.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// A kernel launch with the programmatic stream-serialization attribute (the
// kernel must call pdl_wait() before it reads what the previous kernel wrote).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

// SoA accessors
__device__ __forceinline__ void load3(const float *__restrict__ a, int64_t n, int64_t p, float *o)
{
    o[0] = a[p]; o[1] = a[n + p]; o[2] = a[2 * n + p];
}
__device__ __forceinline__ void store3(float *__restrict__ a, int64_t n, int64_t p, const float *o)
{
    a[p] = o[0]; a[n + p] = o[1]; a[2 * n + p] = o[2];
}
__device__ __forceinline__ void load9(const float *__restrict__ a, int64_t n, int64_t p, float *o)
{
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = a[k * n + p];
}
__device__ __forceinline__ void store9(float *__restrict__ a, int64_t n, int64_t p, const float *o)
{
#pragma unroll
    for (int k = 0; k < 9; ++k) a[k * n + p] = o[k];
}
// symmetric stress, 6 SoA components xx yy zz xy xz yz -> full row-major 3x3
__device__ __forceinline__ void load_sym6(const float *__restrict__ a, int64_t n, int64_t p, float *o)
{
    float xx = a[p], yy = a[n + p], zz = a[2 * n + p], xy = a[3 * n + p], xz = a[4 * n + p], yz = a[5 * n + p];
    o[0] = xx; o[1] = xy; o[2] = xz;
    o[3] = xy; o[4] = yy; o[5] = yz;
    o[6] = xz; o[7] = yz; o[8] = zz;
}
__device__ __forceinline__ void store_sym6(float *__restrict__ a, int64_t n, int64_t p, const float *s)
{
    a[p] = s[0]; a[n + p] = s[4]; a[2 * n + p] = s[8];
    a[3 * n + p] = s[1]; a[4 * n + p] = s[2]; a[5 * n + p] = s[5];
}

}  // namespace mpmw
