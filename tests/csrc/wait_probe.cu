// Test-only probe of the library's bounded mbarrier wait (mpmw_tma.cuh):
// one warp waits on phase 0 of an mbarrier that is either completed at once
// (arrive != 0) or never completed (arrive == 0).  The wait must return false
// after its wall-time bound in the second case, leaving the context usable.
#include "../../mpmwarpydw_b200/csrc/mpmw_tma.cuh"

using namespace mpmw;

__global__ void k_wait_probe(int arrive, unsigned *ok_out, unsigned long long *ns_out)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (arrive && threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 0);  // the only arrival: the phase completes
    const uint64_t t0 = globaltimer_ns();
    const bool ok = mbar_wait_bounded(&bar, 0);
    const uint64_t t1 = globaltimer_ns();
    if (threadIdx.x == 0) {
        *ok_out = ok ? 1u : 0u;
        *ns_out = (unsigned long long)(t1 - t0);
    }
}

// Returns 0 on success (results in *ok and *ns), else the CUDA error code.
extern "C" int wait_probe(int arrive, unsigned *ok, unsigned long long *ns)
{
    unsigned *d_ok = nullptr;
    unsigned long long *d_ns = nullptr;
    cudaError_t e = cudaMalloc(&d_ok, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&d_ns, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        k_wait_probe<<<1, 32>>>(arrive, d_ok, d_ns);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(ok, d_ok, sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(ns, d_ns, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d_ok);
    cudaFree(d_ns);
    return (int)e;
}
