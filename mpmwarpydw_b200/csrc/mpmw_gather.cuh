// mpmw_gather.cuh -- CTA-cooperative grid-to-particle gather (reference:
// utils/mpmRoutines.py:715-802 g2p), shared by the G2P kernel and the fused
// G2P->P2G kernel.
//
// Grid tile: the CTA's stencil bounding box is loaded into shared memory with
// one TMA tensor copy (8x8x8 nodes of float4; nodes outside the grid read as
// zero, which is also what an out-of-grid stencil node contributes here), then
// each particle gathers its 27 nodes from shared memory.  CTAs whose box
// exceeds 8 nodes per axis gather from global memory instead.
//
// Gather: a tensor product -- for each (i, j) the z column is reduced against
// wz, dwz and k*wz, then the (i, j) sums against wy, dwy and j*wy, then against
// wx, dwx and i*wx -- giving
//   v      = sum w g
//   grad v = inv_dx * sum g (x) (dwx wy wz, wx dwy wz, wx wy dwz)
//   C      = 4 inv_dx * (sum w g (x) (i, j, k) - v (x) fx)
// in ~450 fused multiply-adds.
#pragma once
#include "mpmw_common.cuh"
#include "mpmw_math.cuh"
#include "mpmw_tma.cuh"

namespace mpmw {

struct GatherShared {
    float4 tile[kTileNodes];
    uint64_t bar;
    int lo[3], hi[3];
    int tma_ok;
};

// Phase 1 (every thread of the CTA calls it): CTA bounding box of the active
// particles' stencil bases and, when it fits, the TMA load of the grid tile.
// Returns false (uniformly) when the CTA has no active particle.
__device__ __forceinline__ bool gather_prepare(GatherShared &S, bool act, const Weights &W, const CUtensorMap *tmap,
                                               int use_tma, uint32_t *status, bool &tile, int &ox, int &oy, int &oz)
{
    const int t = threadIdx.x;
    if (t < 3) { S.lo[t] = INT32_MAX; S.hi[t] = INT32_MIN; }
    // one read of the status word per CTA, so the tile decision below is uniform:
    // once any CTA has reported a TMA timeout the rest of the launch gathers from
    // global memory
    if (t == 0)
        S.tma_ok = use_tma && !(status && (*reinterpret_cast<volatile uint32_t *>(status) & MPMW_ST_TIMEOUT));
    __syncthreads();
    {
        int lo0 = act ? W.base[0] : INT32_MAX, lo1 = act ? W.base[1] : INT32_MAX, lo2 = act ? W.base[2] : INT32_MAX;
        int hi0 = act ? W.base[0] : INT32_MIN, hi1 = act ? W.base[1] : INT32_MIN, hi2 = act ? W.base[2] : INT32_MIN;
        lo0 = __reduce_min_sync(0xffffffffu, lo0); lo1 = __reduce_min_sync(0xffffffffu, lo1); lo2 = __reduce_min_sync(0xffffffffu, lo2);
        hi0 = __reduce_max_sync(0xffffffffu, hi0); hi1 = __reduce_max_sync(0xffffffffu, hi1); hi2 = __reduce_max_sync(0xffffffffu, hi2);
        if ((t & 31) == 0) {
            atomicMin(&S.lo[0], lo0); atomicMin(&S.lo[1], lo1); atomicMin(&S.lo[2], lo2);
            atomicMax(&S.hi[0], hi0); atomicMax(&S.hi[1], hi1); atomicMax(&S.hi[2], hi2);
        }
    }
    __syncthreads();
    if (S.lo[0] == INT32_MAX) return false;  // no active particle (uniform)
    ox = S.lo[0]; oy = S.lo[1]; oz = S.lo[2];
    tile = S.tma_ok && (int64_t)S.hi[0] - ox + 3 <= kTileEdge && (int64_t)S.hi[1] - oy + 3 <= kTileEdge &&
           (int64_t)S.hi[2] - oz + 3 <= kTileEdge;
    if (tile) {
        if (t == 0) mbar_init(&S.bar, 1);
        __syncthreads();
        if (t == 0) {
            mbar_arrive_expect_tx(&S.bar, kTileBytes);
            tma_load_4d(S.tile, tmap, 0, oz, oy, ox, &S.bar);
        }
        if (!mbar_wait_bounded(&S.bar, 0)) {
            // the copy did not complete: report at once (so later CTAs skip TMA),
            // give it one more bounded wait, and gather from global memory instead
            raise_status(status, MPMW_ST_TIMEOUT);
            mbar_wait_bounded(&S.bar, 0);
            tile = false;
        }
    }
    return true;
}

// Phase 2 (per active particle): the tensor-product gather.
__device__ __forceinline__ void gather_particle(const GatherShared &S, bool tile, int ox, int oy, int oz,
                                                const Weights &W, const mpmw_grid_t &G, float inv_dx, float *nv,
                                                float *nF, float *nC, uint32_t &bad)
{
    const int nx = G.dims[0], ny = G.dims[1], nz = G.dims[2];
    const float4 *__restrict__ gv = reinterpret_cast<const float4 *>(G.v);
    float gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
    float Mi[3] = {0.f, 0.f, 0.f}, Mj[3] = {0.f, 0.f, 0.f}, Mk[3] = {0.f, 0.f, 0.f};
    nv[0] = nv[1] = nv[2] = 0.f;
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
                if (tile) g = S.tile[tb + (i * kTileEdge + j) * kTileEdge + k];
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
}

// F_trial = (I + dt grad v) F = F + dt (grad v F); optional covariance update.
// Fpre: F read ahead (else loaded here).
__device__ __forceinline__ void g2p_deformation(const mpmw_particles_t &P, const mpmw_params_t &prm, int64_t p,
                                                const float *nF, float *Ft, const float *Fpre = nullptr)
{
    const int64_t n = P.n;
    const float dt = prm.dt;
    float F[9];
    if (Fpre) {
#pragma unroll
        for (int k = 0; k < 9; ++k) F[k] = Fpre[k];
    } else {
        load9(P.F, n, p, F);
    }
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
}

}  // namespace mpmw
