// mpmw_noalloc.cu -- a spatial-hash build that needs no device allocation at all.
//
// mpmw_hash_build takes its radix-sort scratch from a workspace the caller
// allocates.  Some callers cannot allocate device memory when they build the
// hash: a host that embeds the solver under a fixed, pre-reserved device-memory
// budget, or a real-time loop where cudaMalloc (which can synchronize the
// device) is not allowed once stepping has started.  mpmw_hash_build_noalloc
// serves them: its scratch is the file-scope device array below, of a fixed
// size chosen for up to MPMW_HASH_NOALLOC_MAX_POINTS points, so the call
// allocates nothing.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and caches it for that
// device.  Make that first call before any stream capture begins.  The cache
// lives as long as the process and does not notice cudaDeviceReset: a reset
// unloads the module, and a later call would pass the stale address.  A caller
// that resets a device must not use this entry point on it afterwards.
//
// Sharing: every call on a device uses the same array.  The array keeps the
// previous call's contents; hash_build overwrites every scratch word it reads
// (keys, histograms, scan blocks) before reading it, and zeroes the cell ranges
// itself, so no clearing is needed between calls.  Two calls whose GPU work
// overlaps (different streams with no ordering between them) race on the array:
// order them on one stream or with events.
#include <mutex>

#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"

namespace {

// hash_workspace_bytes(1 << 20) = 3 x 4 MiB of keys/ids + 2 x 128 KiB of digit
// histograms + the scan's block sums; 13 MiB covers it.
constexpr size_t kNoAllocScratchBytes = 13ull << 20;
static __device__ __align__(256) unsigned char g_hash_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// device address of g_hash_scratch on the current device (looked up once per device)
int scratch_for_current_device(void **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        mpmw::set_error("hash_build_noalloc: no usable current CUDA device");
        return MPMW_E_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_hash_scratch);
        if (e != cudaSuccess || !p) {
            mpmw::set_error("hash_build_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                            cudaGetErrorString(e));
            return MPMW_E_DEVICE;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return MPMW_OK;
}

}  // namespace

extern "C" int mpmw_hash_build_noalloc(const float *x, int64_t n, const mpmw_hash_t *h, mpmw_stream_t stream)
{
    if (n < 0 || n > MPMW_HASH_NOALLOC_MAX_POINTS) {
        mpmw::set_error("hash_build_noalloc: %lld points; this entry point takes 0 to %d (use mpmw_hash_build "
                        "with a caller workspace for more)",
                        (long long)n, MPMW_HASH_NOALLOC_MAX_POINTS);
        return MPMW_E_ARG;
    }
    if (!h) { mpmw::set_error("hash_build_noalloc: NULL hash"); return MPMW_E_ARG; }
    if (n > 0 && !x) { mpmw::set_error("hash_build_noalloc: NULL points"); return MPMW_E_ARG; }
    const size_t need = mpmw::hash_workspace_bytes(n);
    if (need > kNoAllocScratchBytes) {
        mpmw::set_error("hash_build_noalloc: %zu scratch bytes needed, %zu available", need, kNoAllocScratchBytes);
        return MPMW_E_WORKSPACE;
    }
    void *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != MPMW_OK) return rc;
    return mpmw_hash_build(x, n, h, scratch, kNoAllocScratchBytes, stream);
}
