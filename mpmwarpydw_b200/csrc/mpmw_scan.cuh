// mpmw_scan.cuh -- device-wide exclusive prefix sum of int32 counts.
//
// Three launches: per-block scan (kScanBlock elements per CTA) writing block
// totals, one-CTA scan of the block totals (up to kScanBlock * kScanBlock / 1024
// blocks), and a uniform add.  Scratch: (nblocks + 1) int32.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpmw {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;   // 1024 elements per CTA
constexpr int kScanMaxBlocks = kScanThreads * 32;       // single-CTA second level: 8192 blocks

__device__ __forceinline__ int warp_incl_scan(int v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) >= o) v += t;
    }
    return v;
}

// block-wide exclusive scan of one int per thread (blockDim.x == kThreads, a
// multiple of 32 up to 1024); returns the exclusive value and stores the block
// sum in *total in every thread
template <int kThreads = kScanThreads>
__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    constexpr int kWarps = kThreads / 32;
    __shared__ int warp_sums[kWarps + 1];
    int incl = warp_incl_scan(v);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = lane < kWarps ? warp_sums[lane] : 0;
        int si = warp_incl_scan(s);
        if (lane < kWarps) warp_sums[lane] = si - s;
        if (lane == kWarps - 1) warp_sums[kWarps] = si;
    }
    __syncthreads();
    int r = incl - v + warp_sums[wid];
    *total = warp_sums[kWarps];
    __syncthreads();
    return r;
}

// The same scan with one barrier: every warp reads all the warp totals from
// `wsum` (kThreads / 32 ints in shared memory).  The caller must not write
// `wsum` again before its next __syncthreads().
template <int kThreads = kScanThreads>
__device__ __forceinline__ int block_excl_scan_1bar(int v, int *total, int *wsum)
{
    constexpr int kWarps = kThreads / 32;
    const int incl = warp_incl_scan(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    int before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const int s = wsum[w];
        before += w < wid ? s : 0;
        all += s;
    }
    *total = all;
    return before + incl - v;
}

static __global__ void __launch_bounds__(kScanThreads) k_scan_blocks(const int *__restrict__ in, int *__restrict__ out,
                                                             int64_t n, int *__restrict__ block_sums)
{
    __shared__ int s_total;
    int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        sum += v[k];
    }
    int off = block_excl_scan(sum, &s_total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = s_total;
}

// one CTA: exclusive scan of nb block sums in place; writes the grand total to block_sums[nb]
static __global__ void __launch_bounds__(kScanThreads) k_scan_top(int *__restrict__ block_sums, int nb)
{
    __shared__ int s_total;
    const int per = (nb + kScanThreads - 1) / kScanThreads;
    int base = threadIdx.x * per;
    int sum = 0;
    for (int k = 0; k < per; ++k)
        if (base + k < nb) sum += block_sums[base + k];
    int off = block_excl_scan(sum, &s_total);
    for (int k = 0; k < per; ++k)
        if (base + k < nb) {
            int t = block_sums[base + k];
            block_sums[base + k] = off;
            off += t;
        }
    if (threadIdx.x == 0) block_sums[nb] = s_total;
}

static __global__ void __launch_bounds__(kScanThreads) k_scan_add(int *__restrict__ out, int64_t n,
                                                          const int *__restrict__ block_sums)
{
    int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanItems;
    int add = block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] += add;
}

static inline int64_t scan_blocks(int64_t n) { return (n + kScanBlock - 1) / kScanBlock; }

// exclusive scan of n ints; scratch holds scan_blocks(n) + 1 ints; returns false if n is too large
static inline bool exclusive_scan(const int *in, int *out, int64_t n, int *scratch, cudaStream_t s)
{
    int64_t nb = scan_blocks(n);
    if (nb > kScanMaxBlocks) return false;
    if (n == 0) return true;
    k_scan_blocks<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, scratch);
    k_scan_top<<<1, kScanThreads, 0, s>>>(scratch, (int)nb);
    k_scan_add<<<(unsigned)nb, kScanThreads, 0, s>>>(out, n, scratch);
    return true;
}

}  // namespace mpmw
