// mpmw_g2p.cu -- grid-to-particle transfer (reference: utils/mpmRoutines.py:715-802
// g2p + update_cov) and the stress kernels (:229-312).
//
// Grid tile: one CTA handles kBlock consecutive (base-cell sorted) particles.
// The CTA's stencil bounding box is loaded into shared memory with one TMA
// tensor copy (8x8x8 nodes of float4; nodes outside the grid read as zero,
// which is also what an out-of-grid stencil node contributes here), then each
// particle gathers its 27 nodes from shared memory.  CTAs whose box exceeds 8
// nodes per axis gather from global memory instead.
//
// Gather: a tensor product -- for each (i, j) the z column is reduced against
// wz, dwz and k*wz, then the (i, j) sums against wy, dwy and j*wy, then against
// wx, dwx and i*wx -- giving
//   v      = sum w g
//   grad v = inv_dx * sum g (x) (dwx wy wz, wx dwy wz, wx wy dwz)
//   C      = 4 inv_dx * (sum w g (x) (i, j, k) - v (x) fx)
// in ~450 fused multiply-adds.
//
// k_g2p<true> continues, in registers, with the next substep's return map in
// tensor form (mpmw_stress.cuh).  Particles that need the SVD path (large
// deformation, or stress_mode SVD) get their F_trial written and their index
// appended to a worklist; k_stress_list finishes them.  The worklist lives in
// the caller's workspace (mpmw_workspace_bytes).
#include <mutex>
#include <unordered_map>

#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"
#include "mpmw_stress.cuh"
#include "mpmw_tma.cuh"

namespace mpmw {

__global__ void __launch_bounds__(kBlock) k_stress(mpmw_particles_t P, float eff, int mode)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    if (!(P.material[p] <= 1)) return;
    if (P.active[p] != 1) return;
    float Ft[9], Cg[9], Fo[9], out[9];
    load9(P.F_trial, P.n, p, Ft);
    load9(P.C, P.n, p, Cg);
    stress_particle<false>(P, eff, mode, p, Ft, Cg, nullptr, nullptr, Fo, out);
    store9(P.F, P.n, p, Fo);
    store_sym6(P.stress, P.n, p, out);
}

// SVD-path stress for the particles listed by k_g2p<true>
__global__ void __launch_bounds__(kBlock) k_stress_list(mpmw_particles_t P, float eff, const int *__restrict__ list,
                                                       const int *__restrict__ count)
{
    const int cnt = *count;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        const int64_t p = list[q];
        float Ft[9], Cg[9], Fo[9], out[9];
        load9(P.F_trial, P.n, p, Ft);
        load9(P.C, P.n, p, Cg);
        stress_particle<false>(P, eff, MPMW_STRESS_SVD, p, Ft, Cg, nullptr, nullptr, Fo, out);
        store9(P.F, P.n, p, Fo);
        store_sym6(P.stress, P.n, p, out);
    }
}

template <bool Fused>
__global__ void __launch_bounds__(kBlock) k_g2p(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                               uint32_t *status, int *svd_list, int *svd_count,
                                               const __grid_constant__ CUtensorMap tmap, int use_tma)
{
    __shared__ __align__(128) float4 s_tile[kTileNodes];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_lo[3], s_hi[3];
    const int t = threadIdx.x;
    const int64_t n = P.n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + t;
    const int nx = G.dims[0], ny = G.dims[1], nz = G.dims[2];
    if (t < 3) { s_lo[t] = INT32_MAX; s_hi[t] = INT32_MIN; }
    const bool act = p < n && P.active[p] == 1 && P.material[p] <= 1;
    float xp[3] = {0.f, 0.f, 0.f};
    Weights W;
    if (act) {
        load3(P.x, n, p, xp);
        weights(xp, prm.min_bounds, prm.inv_dx, W);
    }
    __syncthreads();
    {
        int lo0 = act ? W.base[0] : INT32_MAX, lo1 = act ? W.base[1] : INT32_MAX, lo2 = act ? W.base[2] : INT32_MAX;
        int hi0 = act ? W.base[0] : INT32_MIN, hi1 = act ? W.base[1] : INT32_MIN, hi2 = act ? W.base[2] : INT32_MIN;
        lo0 = __reduce_min_sync(0xffffffffu, lo0); lo1 = __reduce_min_sync(0xffffffffu, lo1); lo2 = __reduce_min_sync(0xffffffffu, lo2);
        hi0 = __reduce_max_sync(0xffffffffu, hi0); hi1 = __reduce_max_sync(0xffffffffu, hi1); hi2 = __reduce_max_sync(0xffffffffu, hi2);
        if ((t & 31) == 0) {
            atomicMin(&s_lo[0], lo0); atomicMin(&s_lo[1], lo1); atomicMin(&s_lo[2], lo2);
            atomicMax(&s_hi[0], hi0); atomicMax(&s_hi[1], hi1); atomicMax(&s_hi[2], hi2);
        }
    }
    __syncthreads();
    if (s_lo[0] == INT32_MAX) return;  // no active MPM particle (uniform)
    const int ox = s_lo[0], oy = s_lo[1], oz = s_lo[2];
    // once any CTA has reported a TMA timeout the rest of the launch gathers from global memory
    const bool tma_ok = use_tma && !(status && (*reinterpret_cast<volatile uint32_t *>(status) & MPMW_ST_TIMEOUT));
    bool tile = tma_ok && (int64_t)s_hi[0] - ox + 3 <= kTileEdge && (int64_t)s_hi[1] - oy + 3 <= kTileEdge &&
                (int64_t)s_hi[2] - oz + 3 <= kTileEdge;
    uint32_t bad = 0;
    if (tile) {
        if (t == 0) mbar_init(&s_bar, 1);
        __syncthreads();
        if (t == 0) {
            mbar_arrive_expect_tx(&s_bar, kTileBytes);
            tma_load_4d(s_tile, &tmap, 0, oz, oy, ox, &s_bar);
        }
        if (!mbar_wait_bounded(&s_bar, 0)) {
            // the copy did not complete: report at once (so later CTAs skip TMA),
            // give it one more bounded wait, and gather from global memory instead
            raise_status(status, MPMW_ST_TIMEOUT);
            mbar_wait_bounded(&s_bar, 0);
            tile = false;
        }
    }
    if (!act) {
        if (bad) raise_status(status, bad);
        return;
    }
    const float4 *__restrict__ gv = reinterpret_cast<const float4 *>(G.v);
    const float inv_dx = prm.inv_dx, dt = prm.dt;
    float nv[3] = {0.f, 0.f, 0.f}, gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
    float Mi[3] = {0.f, 0.f, 0.f}, Mj[3] = {0.f, 0.f, 0.f}, Mk[3] = {0.f, 0.f, 0.f};
    const bool inside = W.base[0] >= 0 && W.base[1] >= 0 && W.base[2] >= 0 && W.base[0] + 2 < nx &&
                        W.base[1] + 2 < ny && W.base[2] + 2 < nz;
    if (!inside) bad |= MPMW_ST_OOB;
    const int tb = ((W.base[0] - ox) * kTileEdge + (W.base[1] - oy)) * kTileEdge + (W.base[2] - oz);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float SS[3] = {0.f, 0.f, 0.f}, SD[3] = {0.f, 0.f, 0.f}, TS[3] = {0.f, 0.f, 0.f}, US[3] = {0.f, 0.f, 0.f},
              SJ[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float Sv[3] = {0.f, 0.f, 0.f}, Tv[3] = {0.f, 0.f, 0.f}, Uv[3] = {0.f, 0.f, 0.f};
            const int ix = W.base[0] + i, iy = W.base[1] + j;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int iz = W.base[2] + k;
                float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
                if (tile) g = s_tile[tb + (i * kTileEdge + j) * kTileEdge + k];
                else if (inside || (ix >= 0 && iy >= 0 && iz >= 0 && ix < nx && iy < ny && iz < nz))
                    g = __ldg(&gv[((int64_t)ix * ny + iy) * nz + iz]);
                const float wz = W.w[2][k], dwz = W.dw[2][k], kwz = (float)k * wz;
                Sv[0] = fma_(wz, g.x, Sv[0]); Sv[1] = fma_(wz, g.y, Sv[1]); Sv[2] = fma_(wz, g.z, Sv[2]);
                Tv[0] = fma_(dwz, g.x, Tv[0]); Tv[1] = fma_(dwz, g.y, Tv[1]); Tv[2] = fma_(dwz, g.z, Tv[2]);
                Uv[0] = fma_(kwz, g.x, Uv[0]); Uv[1] = fma_(kwz, g.y, Uv[1]); Uv[2] = fma_(kwz, g.z, Uv[2]);
            }
            const float wy = W.w[1][j], dwy = W.dw[1][j], jwy = (float)j * wy;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                SS[r] = fma_(wy, Sv[r], SS[r]);
                SD[r] = fma_(dwy, Sv[r], SD[r]);
                TS[r] = fma_(wy, Tv[r], TS[r]);
                US[r] = fma_(wy, Uv[r], US[r]);
                SJ[r] = fma_(jwy, Sv[r], SJ[r]);
            }
        }
        const float wx = W.w[0][i], dwx = W.dw[0][i], iwx = (float)i * wx;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            nv[r] = fma_(wx, SS[r], nv[r]);
            gx[r] = fma_(dwx, SS[r], gx[r]);
            gy[r] = fma_(wx, SD[r], gy[r]);
            gz[r] = fma_(wx, TS[r], gz[r]);
            Mi[r] = fma_(iwx, SS[r], Mi[r]);
            Mj[r] = fma_(wx, SJ[r], Mj[r]);
            Mk[r] = fma_(wx, US[r], Mk[r]);
        }
    }
    float nF[9], nC[9];
    const float c4 = 4.f * inv_dx;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        nF[3 * r + 0] = gx[r] * inv_dx;
        nF[3 * r + 1] = gy[r] * inv_dx;
        nF[3 * r + 2] = gz[r] * inv_dx;
        nC[3 * r + 0] = c4 * fma_(-W.fx[0], nv[r], Mi[r]);
        nC[3 * r + 1] = c4 * fma_(-W.fx[1], nv[r], Mj[r]);
        nC[3 * r + 2] = c4 * fma_(-W.fx[2], nv[r], Mk[r]);
    }
    float xn[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xn[a] = fma_(dt, nv[a], xp[a]);
    if (!(isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]))) bad |= MPMW_ST_NAN;
    float F[9], Ft[9];
    load9(P.F, n, p, F);
    // F_trial = (I + dt grad v) F = F + dt (grad v F)
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float gf = fma_(nF[3 * r + 0], F[c], fma_(nF[3 * r + 1], F[3 + c], nF[3 * r + 2] * F[6 + c]));
            Ft[3 * r + c] = fma_(dt, gf, F[3 * r + c]);
        }
    if (prm.update_cov && P.cov) {
        float *cv = P.cov + 6 * p;
        float cn[9] = {cv[0], cv[1], cv[2], cv[1], cv[3], cv[4], cv[2], cv[4], cv[5]};
        float a1[9], a2[9];
        matmul3(nF, cn, a1);
        matmul3_bt(cn, nF, a2);
        float c1[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) c1[q] = fma_(dt, a1[q] + a2[q], cn[q]);
        cv[0] = c1[0]; cv[1] = c1[1]; cv[2] = c1[2]; cv[3] = c1[4]; cv[4] = c1[5]; cv[5] = c1[8];
    }
    store3(P.x, n, p, xn);
    store9(P.C, n, p, nC);
    if (Fused) {
        float Fo[9], T[9];
        if (prm.stress_mode == MPMW_STRESS_AUTO && small_strain_update<true>(P, prm.eff, p, Ft, xn, nv, Fo, T)) {
            float out[9];
            add_viscous(T, nC, P.eta_shear[p], P.eta_bulk[p], out);
            store9(P.F, n, p, Fo);
            store_sym6(P.stress, n, p, out);
        } else {
            store9(P.F_trial, n, p, Ft);
            svd_list[atomicAdd(svd_count, 1)] = (int)p;
        }
    } else {
        store9(P.F_trial, n, p, Ft);
    }
    store3(P.v, n, p, nv);
    if (bad) raise_status(status, bad);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// cuTensorMapEncodeTiled is a driver API call; it is resolved through the
// runtime (cudaGetDriverEntryPoint) so that libmpmw.so does not link libcuda
// and loads on machines without a GPU driver.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiledFn>(f);
    }();
    return fn;
}

bool grid_tensor_map(const float *base, const int *dims, CUtensorMap *out)
{
    EncodeTiledFn encode = encode_tiled_fn();
    if (!encode) return false;
    cuuint64_t gdim[4] = {4, (cuuint64_t)dims[2], (cuuint64_t)dims[1], (cuuint64_t)dims[0]};
    cuuint64_t gstride[3] = {16, (cuuint64_t)dims[2] * 16, (cuuint64_t)dims[1] * dims[2] * 16};
    cuuint32_t box[4] = {4, kTileEdge, kTileEdge, kTileEdge};
    cuuint32_t estride[4] = {1, 1, 1, 1};
    CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(base), gdim, gstride, box,
                        estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

namespace {
struct MapKey {
    const float *p;
    int d0, d1, d2;
    bool operator==(const MapKey &o) const { return p == o.p && d0 == o.d0 && d1 == o.d1 && d2 == o.d2; }
};
struct MapKeyHash {
    size_t operator()(const MapKey &k) const
    {
        return std::hash<const void *>()(k.p) ^ ((size_t)k.d0 * 73856093u) ^ ((size_t)k.d1 * 19349663u) ^
               ((size_t)k.d2 * 83492791u);
    }
};
std::mutex g_map_mu;
std::unordered_map<MapKey, CUtensorMap, MapKeyHash> g_maps;
}  // namespace

// cached tensor map of grid.v; false if TMA cannot describe it
static bool cached_grid_map(const mpmw_grid_t &g, CUtensorMap *out)
{
    MapKey key{g.v, g.dims[0], g.dims[1], g.dims[2]};
    std::lock_guard<std::mutex> lk(g_map_mu);
    auto it = g_maps.find(key);
    if (it != g_maps.end()) { *out = it->second; return true; }
    CUtensorMap m;
    if (!grid_tensor_map(g.v, g.dims, &m)) return false;
    if (g_maps.size() > 64) g_maps.clear();
    g_maps.emplace(key, m);
    *out = m;
    return true;
}

size_t g2p_workspace_bytes(int64_t n) { return (size_t)(256 + ((n * 4 + 255) / 256) * 256); }

int launch_stress(const mpmw_particles_t &p, const mpmw_params_t &prm, cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    k_stress<<<grid_for(p.n), kBlock, 0, s>>>(p, prm.eff, prm.stress_mode);
    return check_launch("k_stress");
}

int launch_g2p(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, bool fused,
               void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    CUtensorMap map;
    int use_tma = cached_grid_map(g, &map) ? 1 : 0;
    if (!use_tma) memset(&map, 0, sizeof(map));
    if (!fused) {
        k_g2p<false><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st, nullptr, nullptr, map, use_tma);
        return check_launch("k_g2p");
    }
    if (!ws || ws_bytes < g2p_workspace_bytes(p.n)) {
        set_error("g2p_stress: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  g2p_workspace_bytes(p.n));
        return MPMW_E_WORKSPACE;
    }
    int *count = static_cast<int *>(ws);
    int *list = reinterpret_cast<int *>(static_cast<char *>(ws) + 256);
    if (cudaMemsetAsync(count, 0, sizeof(int), s) != cudaSuccess) { set_error("g2p_stress: memset failed"); return MPMW_E_DEVICE; }
    k_g2p<true><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st, list, count, map, use_tma);
    MPMW_TRY_LAUNCH("k_g2p<fused>");
    k_stress_list<<<148 * 4, kBlock, 0, s>>>(p, prm.eff, list, count);
    return check_launch("k_stress_list");
}

}  // namespace mpmw
