// mpmw_g2p.cu -- grid-to-particle transfer (reference: utils/mpmRoutines.py:715-802
// g2p + update_cov) and the stress kernel (:229-312).
//
// The 27-node gather is evaluated as a tensor product: for each (i, j) the z
// column is reduced against wz, dwz and k*wz, then the (i, j) sums against wy,
// dwy and j*wy, then against wx, dwx and i*wx.  That yields
//   v      = sum w g
//   grad v = inv_dx * sum g (x) (dwx wy wz, wx dwy wz, wx wy dwz)
//   C      = 4 inv_dx * (sum w g (x) (i, j, k) - v (x) fx)
// in ~450 fused multiply-adds instead of ~2000 separate operations.
// k_g2p<true> continues, in registers, with the next substep's return map.
#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"
#include "mpmw_stress.cuh"

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

template <bool Fused>
__global__ void __launch_bounds__(kBlock) k_g2p(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                               uint32_t *status)
{
    const int64_t n = P.n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (P.active[p] != 1) return;
    if (!(P.material[p] <= 1)) return;
    const int nx = G.dims[0], ny = G.dims[1], nz = G.dims[2];
    const float4 *__restrict__ gv = reinterpret_cast<const float4 *>(G.v);
    float xp[3];
    load3(P.x, n, p, xp);
    Weights W;
    weights(xp, prm.min_bounds, prm.inv_dx, W);
    const float inv_dx = prm.inv_dx, dt = prm.dt;
    float nv[3] = {0.f, 0.f, 0.f}, gx[3] = {0.f, 0.f, 0.f}, gy[3] = {0.f, 0.f, 0.f}, gz[3] = {0.f, 0.f, 0.f};
    float Mi[3] = {0.f, 0.f, 0.f}, Mj[3] = {0.f, 0.f, 0.f}, Mk[3] = {0.f, 0.f, 0.f};
    uint32_t bad = 0;
    const bool inside = W.base[0] >= 0 && W.base[1] >= 0 && W.base[2] >= 0 && W.base[0] + 2 < nx &&
                        W.base[1] + 2 < ny && W.base[2] + 2 < nz;
    if (!inside) bad = MPMW_ST_OOB;
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
                if (inside || (ix >= 0 && iy >= 0 && iz >= 0 && ix < nx && iy < ny && iz < nz))
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
        float Fo[9], out[9];
        stress_particle<true>(P, prm.eff, prm.stress_mode, p, Ft, nC, xn, nv, Fo, out);
        store9(P.F, n, p, Fo);
        store_sym6(P.stress, n, p, out);
    } else {
        store9(P.F_trial, n, p, Ft);
    }
    store3(P.v, n, p, nv);
    if (bad) raise_status(status, bad);
}

int launch_stress(const mpmw_particles_t &p, const mpmw_params_t &prm, cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    k_stress<<<grid_for(p.n), kBlock, 0, s>>>(p, prm.eff, prm.stress_mode);
    return check_launch("k_stress");
}

int launch_g2p(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, bool fused,
               cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    if (fused) k_g2p<true><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st);
    else k_g2p<false><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st);
    return check_launch(fused ? "k_g2p<fused>" : "k_g2p");
}

}  // namespace mpmw
