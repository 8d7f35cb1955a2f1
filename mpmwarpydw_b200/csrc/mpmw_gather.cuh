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

constexpr int kGatherMaxWarps = 8;  // warps of a gathering CTA (256 threads)

struct GatherShared {
    float4 tile[kTileNodes];
    uint64_t bar;
    int lo[3], hi[3];
    int wbox[kGatherMaxWarps][6];  // each warp's min and max stencil base (one barrier, no atomics)
    int tma_ok;
};

// Phase 1 (every thread of the CTA calls it): CTA bounding box of the active
// particles' stencil bases and, when it fits, the TMA load of the grid tile.
// Returns false (uniformly) when the CTA has no active particle.  tmap is a
// kernel parameter (or an element of one).
__device__ __forceinline__ bool gather_prepare(GatherShared &S, bool act, const Weights &W, const CUtensorMap *tmap,
                                               int use_tma, uint32_t *status, bool &tile, int &ox, int &oy, int &oz)
{
    const int t = threadIdx.x, lane = t & 31, nw = (int)(blockDim.x >> 5);
    // one read of the status word per CTA, so the tile decision below is uniform:
    // once any CTA has reported a TMA timeout the rest of the launch gathers from
    // global memory
    if (t == 0) {
        S.tma_ok = use_tma && !(status && (*reinterpret_cast<volatile uint32_t *>(status) & MPMW_ST_TIMEOUT));
        mbar_init(&S.bar, 1);  // used only if the tile fits; the barrier below publishes it
    }
    {
        // each warp's box into its own slot (no initialisation, no atomics) ...
        int lo0 = act ? W.base[0] : INT32_MAX, lo1 = act ? W.base[1] : INT32_MAX, lo2 = act ? W.base[2] : INT32_MAX;
        int hi0 = act ? W.base[0] : INT32_MIN, hi1 = act ? W.base[1] : INT32_MIN, hi2 = act ? W.base[2] : INT32_MIN;
        lo0 = __reduce_min_sync(0xffffffffu, lo0); lo1 = __reduce_min_sync(0xffffffffu, lo1); lo2 = __reduce_min_sync(0xffffffffu, lo2);
        hi0 = __reduce_max_sync(0xffffffffu, hi0); hi1 = __reduce_max_sync(0xffffffffu, hi1); hi2 = __reduce_max_sync(0xffffffffu, hi2);
        if (lane == 0) {
            int *w = S.wbox[t >> 5];
            w[0] = lo0; w[1] = lo1; w[2] = lo2; w[3] = hi0; w[4] = hi1; w[5] = hi2;
        }
    }
    __syncthreads();
    int b[6];
    {
        // ... then every warp reduces the slots: lane w reads warp w's
#pragma unroll
        for (int c = 0; c < 6; ++c) b[c] = lane < nw ? S.wbox[lane][c] : (c < 3 ? INT32_MAX : INT32_MIN);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            b[c] = __reduce_min_sync(0xffffffffu, b[c]);
            b[c + 3] = __reduce_max_sync(0xffffffffu, b[c + 3]);
        }
    }
    // the box for the caller (the fused kernel's scatter reads it with no
    // barrier in between): every thread stores the same values, so each thread
    // reads back its own store or an identical one
#pragma unroll
    for (int c = 0; c < 3; ++c) { S.lo[c] = b[c]; S.hi[c] = b[c + 3]; }
    if (b[0] == INT32_MAX) return false;  // no active particle (uniform)
    ox = b[0]; oy = b[1]; oz = b[2];
    tile = S.tma_ok && (int64_t)b[3] - ox + 3 <= kTileEdge && (int64_t)b[4] - oy + 3 <= kTileEdge &&
           (int64_t)b[5] - oz + 3 <= kTileEdge;
    if (tile) {
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

// Phase 2 (per active particle): the tensor-product gather.  The x and y
// components share every weight, so they are summed as float2 pairs with the
// packed FP32 FMA (__ffma2_rn: two FMAs, each rounded once, in one
// instruction); the z component is summed alone.  Same operations and
// rounding as three scalar FMAs.  The moment sums (i, j, k times the weight)
// skip the terms whose factor is exactly 0: for finite grid velocities they
// add +-0 and leave the sum unchanged.
__device__ __forceinline__ float2 ffma2(float w, float2 g, float2 acc) { return __ffma2_rn(make_float2(w, w), g, acc); }

// Tile: the CTA's grid tile is in shared memory (a uniform choice, made once
// per CTA, so the 27 node reads compile without a branch each).
template <bool Tile>
__device__ __forceinline__ void gather_particle_t(const GatherShared &S, int ox, int oy, int oz, const Weights &W,
                                                  const mpmw_grid_t &G, float inv_dx, float *nv, float *nF, float *nC,
                                                  uint32_t &bad)
{
    const int nx = G.dims[0], ny = G.dims[1], nz = G.dims[2];
    const float4 *__restrict__ gv = reinterpret_cast<const float4 *>(G.v);
    float2 v2 = make_float2(0.f, 0.f), gx2 = v2, gy2 = v2, gz2 = v2, Mi2 = v2, Mj2 = v2, Mk2 = v2;
    float vz = 0.f, gxz = 0.f, gyz = 0.f, gzz = 0.f, Miz = 0.f, Mjz = 0.f, Mkz = 0.f;
    const bool inside = W.base[0] >= 0 && W.base[1] >= 0 && W.base[2] >= 0 && W.base[0] + 2 < nx &&
                        W.base[1] + 2 < ny && W.base[2] + 2 < nz;
    if (!inside) bad |= MPMW_ST_OOB;
    const int tb = ((W.base[0] - ox) * kTileEdge + (W.base[1] - oy)) * kTileEdge + (W.base[2] - oz);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float2 SS2 = make_float2(0.f, 0.f), SD2 = SS2, TS2 = SS2, US2 = SS2, SJ2 = SS2;
        float SSz = 0.f, SDz = 0.f, TSz = 0.f, USz = 0.f, SJz = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float2 Sv2 = make_float2(0.f, 0.f), Tv2 = Sv2, Uv2 = Sv2;
            float Svz = 0.f, Tvz = 0.f, Uvz = 0.f;
            const int ix = W.base[0] + i, iy = W.base[1] + j;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int iz = W.base[2] + k;
                float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
                if (Tile) g = S.tile[tb + (i * kTileEdge + j) * kTileEdge + k];
                else if (inside || (ix >= 0 && iy >= 0 && iz >= 0 && ix < nx && iy < ny && iz < nz))
                    g = __ldg(&gv[((int64_t)ix * ny + iy) * nz + iz]);
                const float wz = W.w[2][k], dwz = W.dw[2][k], kwz = (float)k * wz;
                const float2 gxy = make_float2(g.x, g.y);
                Sv2 = ffma2(wz, gxy, Sv2); Svz = fma_(wz, g.z, Svz);
                Tv2 = ffma2(dwz, gxy, Tv2); Tvz = fma_(dwz, g.z, Tvz);
                if (k > 0) { Uv2 = ffma2(kwz, gxy, Uv2); Uvz = fma_(kwz, g.z, Uvz); }  // k = 0 adds 0 * g
            }
            const float wy = W.w[1][j], dwy = W.dw[1][j], jwy = (float)j * wy;
            SS2 = ffma2(wy, Sv2, SS2); SSz = fma_(wy, Svz, SSz);
            SD2 = ffma2(dwy, Sv2, SD2); SDz = fma_(dwy, Svz, SDz);
            TS2 = ffma2(wy, Tv2, TS2); TSz = fma_(wy, Tvz, TSz);
            US2 = ffma2(wy, Uv2, US2); USz = fma_(wy, Uvz, USz);
            if (j > 0) { SJ2 = ffma2(jwy, Sv2, SJ2); SJz = fma_(jwy, Svz, SJz); }  // j = 0 adds 0 * Sv
        }
        const float wx = W.w[0][i], dwx = W.dw[0][i], iwx = (float)i * wx;
        v2 = ffma2(wx, SS2, v2); vz = fma_(wx, SSz, vz);
        gx2 = ffma2(dwx, SS2, gx2); gxz = fma_(dwx, SSz, gxz);
        gy2 = ffma2(wx, SD2, gy2); gyz = fma_(wx, SDz, gyz);
        gz2 = ffma2(wx, TS2, gz2); gzz = fma_(wx, TSz, gzz);
        if (i > 0) { Mi2 = ffma2(iwx, SS2, Mi2); Miz = fma_(iwx, SSz, Miz); }  // i = 0 adds 0 * SS
        Mj2 = ffma2(wx, SJ2, Mj2); Mjz = fma_(wx, SJz, Mjz);
        Mk2 = ffma2(wx, US2, Mk2); Mkz = fma_(wx, USz, Mkz);
    }
    nv[0] = v2.x; nv[1] = v2.y; nv[2] = vz;
    const float gx[3] = {gx2.x, gx2.y, gxz}, gy[3] = {gy2.x, gy2.y, gyz}, gz[3] = {gz2.x, gz2.y, gzz};
    const float Mi[3] = {Mi2.x, Mi2.y, Miz}, Mj[3] = {Mj2.x, Mj2.y, Mjz}, Mk[3] = {Mk2.x, Mk2.y, Mkz};
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

__device__ __forceinline__ void gather_particle(const GatherShared &S, bool tile, int ox, int oy, int oz,
                                                const Weights &W, const mpmw_grid_t &G, float inv_dx, float *nv,
                                                float *nF, float *nC, uint32_t &bad)
{
    if (tile) gather_particle_t<true>(S, ox, oy, oz, W, G, inv_dx, nv, nF, nC, bad);
    else gather_particle_t<false>(S, ox, oy, oz, W, G, inv_dx, nv, nF, nC, bad);
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
