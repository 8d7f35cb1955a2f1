// mpmw_p2g.cu -- APIC particle-to-grid transfer with stress (reference:
// utils/mpmRoutines.py:485-569 p2g_apic_with_stress): one CTA per chunk of
// kScatterChunk consecutive particles, scattered by p2g_scatter
// (mpmw_scatter.cuh).
#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"
#include "mpmw_scatter.cuh"

namespace mpmw {

__global__ void __launch_bounds__(kScatterChunk) k_p2g(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                       uint32_t *status)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ScatterShared &S = *reinterpret_cast<ScatterShared *>(smem_raw);
    const int64_t n = P.n;
    const int64_t p = (int64_t)blockIdx.x * kScatterChunk + threadIdx.x;
    // labels and the particle's fields are loaded together (not behind the label test)
    int lab_a = 0, lab_m = 0;
    float xp[3] = {0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f}, C0[9], st6[6];
    float m = 0.f, vol = 0.f;
    if (p < n) {
        lab_a = P.active[p];
        lab_m = P.material[p];
        load3(P.x, n, p, xp);
        load3(P.v, n, p, v);
        load9(P.C, n, p, C0);
#pragma unroll
        for (int e = 0; e < 6; ++e) st6[e] = P.stress[(int64_t)e * n + p];
        m = P.mass[p];
        vol = P.vol[p];
    }
    const bool act = lab_a == 1 && lab_m <= 1;
    uint32_t bad = 0;
    p2g_scatter(S, act, xp, v, C0, st6, m, vol, prm, reinterpret_cast<float4 *>(G.mv), G.dims[0], G.dims[1],
                G.dims[2], bad);
    if (bad) raise_status(status, bad);
}

static bool g_p2g_attr[64];

int launch_p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_error("p2g: no current device"); return MPMW_E_DEVICE; }
    const size_t smem = sizeof(ScatterShared);
    if (dev >= 0 && dev < 64 && !g_p2g_attr[dev]) {
        if (cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
            set_error("p2g: cannot reserve %zu bytes of shared memory", smem);
            return MPMW_E_DEVICE;
        }
        g_p2g_attr[dev] = true;
    }
    k_p2g<<<grid_for(p.n, kScatterChunk), kScatterChunk, smem, s>>>(p, g, prm, st);
    return check_launch("k_p2g");
}

}  // namespace mpmw
