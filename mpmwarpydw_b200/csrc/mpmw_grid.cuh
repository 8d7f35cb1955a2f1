// mpmw_grid.cuh -- the grid pass of a substep, per node (reference:
// utils/mpmRoutines.py:690-711 normalisation, gravity and damping, and the
// boundary kernels at :914-1362), shared by the single-scene and batched
// grid-update kernels.
#pragma once
#include "mpmw_common.cuh"
#include "mpmw_math.cuh"

namespace mpmw {

__device__ __forceinline__ float coulomb(float v, float mu, float dt, float g)
{
    if (fabsf(v) < 1e-12f) return 0.f;
    float dvf = (mu * g) * dt;
    float s = v < 0.f ? -1.f : 1.f;
    return s * rmax(fabsf(v) - dvf, 0.f);
}

__device__ __forceinline__ void apply_bc(int bc, const int *idx, const int *dim, float *o, float mu, float rest,
                                         float dt, float g, int pad)
{
    float v[3] = {o[0], o[1], o[2]};
    if (bc == MPMW_BC_FRICTION || bc == MPMW_BC_RESTITUTION) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int t0 = (a + 1) % 3, t1 = (a + 2) % 3;
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                bool hit = side == 0 ? (idx[a] <= pad && v[a] < 0.f) : (idx[a] >= dim[a] - pad && v[a] > 0.f);
                if (!hit) continue;
                float w[3];
                w[a] = bc == MPMW_BC_FRICTION ? 0.f : -rest * v[a];
                w[t0] = coulomb(v[t0], mu, dt, g);
                w[t1] = coulomb(v[t1], mu, dt, g);
                o[0] = w[0]; o[1] = w[1]; o[2] = w[2];
            }
        }
    } else if (bc == MPMW_BC_FRICTION_GRADUAL) {
        const float padf = (float)pad;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int t0 = (a + 1) % 3, t1 = (a + 2) % 3;
            float fade = 0.f;
            bool hit = false;
            if (idx[a] < pad && v[a] < 0.f) { fade = (float)idx[a] / padf; hit = true; }
            else if (idx[a] >= dim[a] - pad && v[a] > 0.f) { fade = (float)(dim[a] - 1 - idx[a]) / padf; hit = true; }
            if (!hit) continue;
            float fm = mu * (1.f - fade);
            float w[3];
            w[t0] = coulomb(v[t0], fm, dt, g);
            w[t1] = coulomb(v[t1], fm, dt, g);
            w[a] = 0.f * (1.f - fade) + v[a] * fade;
            o[0] = w[0]; o[1] = w[1]; o[2] = w[2];
        }
    } else if (bc == MPMW_BC_ABSORBING) {
        const float padf = (float)pad;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                bool hit = side == 0 ? (idx[a] < 3) : (idx[a] >= dim[a] - 3);
                if (!hit) continue;
                float lf = side == 0 ? (padf - (float)idx[a]) / padf : (padf - (float)(dim[a] - 1 - idx[a])) / padf;
                float damp = 0.f * lf + 1.f * (1.f - lf);
                o[0] = v[0] * damp; o[1] = v[1] * damp; o[2] = v[2] * damp;
            }
        }
    } else if (bc == MPMW_BC_PLANE_STRAIN_Y) {
        const int ix = idx[0], iy = idx[1], iz = idx[2];
        if (ix <= pad && v[0] < 0.f) { o[0] = 0.f; o[1] = coulomb(v[1], mu, dt, g); o[2] = coulomb(v[2], mu, dt, g); }
        if (ix >= dim[0] - pad && v[0] > 0.f) { o[0] = 0.f; o[1] = coulomb(v[1], mu, dt, g); o[2] = coulomb(v[2], mu, dt, g); }
        if (iy <= pad) { v[0] = o[0]; v[1] = o[1]; v[2] = o[2]; o[0] = v[0]; o[1] = 0.f; o[2] = v[2]; }
        if (iy >= dim[1] - pad) { v[0] = o[0]; v[1] = o[1]; v[2] = o[2]; o[0] = v[0]; o[1] = 0.f; o[2] = v[2]; }
        if (iz <= pad && v[2] < 0.f) { float a0 = coulomb(v[0], mu, dt, g), a1 = coulomb(v[1], mu, dt, g); o[0] = a0; o[1] = a1; o[2] = 0.f; }
        if (iz >= dim[2] - pad && v[2] > 0.f) { float a0 = coulomb(v[0], mu, dt, g), a1 = coulomb(v[1], mu, dt, g); o[0] = a0; o[1] = a1; o[2] = 0.f; }
    } else if (bc == MPMW_BC_PLANE_STRAIN_Y_GLOBAL) {
        const int ix = idx[0], iz = idx[2];
        o[1] = 0.f;
        v[0] = o[0]; v[1] = o[1]; v[2] = o[2];
        if (ix <= pad && v[0] < 0.f) { o[0] = 0.f; o[1] = 0.f; o[2] = coulomb(v[2], mu, dt, g); }
        if (ix >= dim[0] - pad && v[0] > 0.f) { o[0] = 0.f; o[1] = 0.f; o[2] = coulomb(v[2], mu, dt, g); }
        if (iz <= pad && v[2] < 0.f) { o[0] = coulomb(v[0], mu, dt, g); o[1] = 0.f; o[2] = 0.f; }
        if (iz >= dim[2] - pad && v[2] > 0.f) { o[0] = coulomb(v[0], mu, dt, g); o[1] = 0.f; o[2] = 0.f; }
    }
}

// The grid update of node g (inside the grid) whose accumulators (m, m v)
// were read as `a`.  zero_mv: also clear the accumulators (for the fused
// G2P->P2G kernel, which scatters the next substep into them).
__device__ __forceinline__ void grid_update_apply(const mpmw_grid_t &G, const mpmw_params_t &prm, int zero_mv,
                                                  int64_t g, const float4 a)
{
    const int ny = G.dims[1], nz = G.dims[2];
    if (zero_mv) reinterpret_cast<float4 *>(G.mv)[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    float o[3] = {0.f, 0.f, 0.f};
    if (a.x > 1e-15f) {
        float inv = 1.f / a.x;
        o[0] = a.y * inv + prm.dt * prm.gravity[0];
        o[1] = a.z * inv + prm.dt * prm.gravity[1];
        o[2] = a.w * inv + prm.dt * prm.gravity[2];
    }
    if (prm.grid_v_damping_scale < 1.f) {
        o[0] = o[0] * prm.grid_v_damping_scale;
        o[1] = o[1] * prm.grid_v_damping_scale;
        o[2] = o[2] * prm.grid_v_damping_scale;
    }
    if (prm.boundary_condition >= 0) {
        // node coordinates in 32-bit arithmetic: grids hold at most 2^31 - 1
        // nodes (checked on the host), and 64-bit division is a long routine
        const int gi = (int)g;
        const int iz = gi % nz, r = gi / nz;
        const int iy = r % ny, ix = r / ny;
        int idx[3] = {ix, iy, iz}, dim[3] = {G.dims[0], ny, nz};
        float gm = fabsf(prm.gravity[2]);
        apply_bc(prm.boundary_condition, idx, dim, o, prm.bound_friction, prm.bound_restitution, prm.dt, gm,
                 prm.boundary_padding);
    }
    reinterpret_cast<float4 *>(G.v)[g] = make_float4(o[0], o[1], o[2], 0.f);
}

// One node g of the grid update (g beyond the grid returns).
__device__ __forceinline__ void grid_update_node(const mpmw_grid_t &G, const mpmw_params_t &prm, int zero_mv, int64_t g)
{
    if (g >= (int64_t)G.dims[0] * G.dims[1] * G.dims[2]) return;
    grid_update_apply(G, prm, zero_mv, g, reinterpret_cast<const float4 *>(G.mv)[g]);
}

}  // namespace mpmw
