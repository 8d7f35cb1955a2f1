// mpmw_mpm.cu -- MPM substep kernels and their C-ABI entry points.
//
// Kernel map (reference = MPMWarpYDW utils/...):
//   (k_stress, k_g2p: mpmw_g2p.cu; k_p2g: mpmw_p2g.cu)
//   k_grid_update  mpmRoutines.py:690-711 + boundary kernels :914-1362, one pass
//   k_vlc_*        mpmRoutines.py:817-911
#include <cstdarg>
#include <cstring>

#include "mpmw_common.cuh"
#include "mpmw_grid.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"

namespace mpmw {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return MPMW_E_LAUNCH;
    }
    return MPMW_OK;
}

// zero_mv: also clear the accumulators after reading them (for the fused
// G2P->P2G kernel, which scatters the next substep into them).
// reset (may be NULL): set to 0 once, for the fused kernel's worklist count.
__global__ void __launch_bounds__(kBlock) k_grid_update(mpmw_grid_t G, mpmw_params_t prm, int zero_mv, int *reset)
{
    pdl_wait();
    pdl_trigger();
    if (reset && blockIdx.x == 0 && threadIdx.x == 0) *reset = 0;
    grid_update_node(G, prm, zero_mv, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// single grid operations with the reference kernels' exact write sets:
//   op 0: grid_normalization_and_gravity (writes only nodes with m > 1e-15)
//   op 1: add_damping_via_grid (unconditional scale)
//   op 2: the boundary kernel prm.boundary_condition on grid v
__global__ void __launch_bounds__(kBlock) k_grid_op(mpmw_grid_t G, mpmw_params_t prm, int op)
{
    const int nx = G.dims[0], ny = G.dims[1], nz = G.dims[2];
    const int64_t total = (int64_t)nx * ny * nz;
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    float4 *v4 = reinterpret_cast<float4 *>(G.v);
    if (op == 0) {
        const float4 a = reinterpret_cast<const float4 *>(G.mv)[g];
        if (a.x > 1e-15f) {
            float inv = 1.f / a.x;
            v4[g] = make_float4(a.y * inv + prm.dt * prm.gravity[0], a.z * inv + prm.dt * prm.gravity[1],
                                a.w * inv + prm.dt * prm.gravity[2], 0.f);
        }
    } else if (op == 1) {
        float4 t = v4[g];
        float s = prm.grid_v_damping_scale;
        v4[g] = make_float4(t.x * s, t.y * s, t.z * s, t.w);
    } else {
        float4 t = v4[g];
        float o[3] = {t.x, t.y, t.z};
        const int gi = (int)g;  // grids hold at most 2^31 - 1 nodes
        int iz = gi % nz, r = gi / nz;
        int iy = r % ny, ix = r / ny;
        int idx[3] = {ix, iy, iz}, dim[3] = {nx, ny, nz};
        apply_bc(prm.boundary_condition, idx, dim, o, prm.bound_friction, prm.bound_restitution, prm.dt,
                 fabsf(prm.gravity[2]), prm.boundary_padding);
        v4[g] = make_float4(o[0], o[1], o[2], t.w);
    }
}

// ---------------------------------------------------------------------------
// volumetric locking correction
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool vlc_cell(const float *xp, const mpmw_params_t &prm, const int *dims, int64_t &cell)
{
    int c0 = (int)((xp[0] - prm.min_bounds[0]) * prm.inv_dx);
    int c1 = (int)((xp[1] - prm.min_bounds[1]) * prm.inv_dx);
    int c2 = (int)((xp[2] - prm.min_bounds[2]) * prm.inv_dx);
    if (c0 < 0 || c1 < 0 || c2 < 0 || c0 >= dims[0] || c1 >= dims[1] || c2 >= dims[2]) return false;
    cell = ((int64_t)c0 * dims[1] + c1) * dims[2] + c2;
    return true;
}

__global__ void __launch_bounds__(kBlock) k_vlc_acc(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                   uint32_t *status)
{
    const int64_t n = P.n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (!(P.active[p] == 1 && P.material[p] <= 1)) return;
    float xp[3];
    load3(P.x, n, p, xp);
    int64_t cell;
    if (!vlc_cell(xp, prm, G.dims, cell)) { raise_status(status, MPMW_ST_OOB); return; }
    float div = (P.C[p] + P.C[4 * n + p]) + P.C[8 * n + p];
    float vp = P.vol[p];
    atomicAdd(&G.cell_div[cell], div * vp);
    atomicAdd(&G.cell_vol[cell], vp);
}

__global__ void __launch_bounds__(kBlock) k_vlc_apply(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                     uint32_t *status)
{
    const int64_t n = P.n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (!(P.active[p] == 1 && P.material[p] <= 1)) return;
    float xp[3];
    load3(P.x, n, p, xp);
    int64_t cell;
    float vs = 0.f, cd = 0.f;
    if (!vlc_cell(xp, prm, G.dims, cell)) raise_status(status, MPMW_ST_OOB);
    else { vs = G.cell_vol[cell]; cd = G.cell_div[cell]; }
    float dvc = vs > 1e-20f ? cd / vs : 0.f;
    float c00 = P.C[p], c11 = P.C[4 * n + p], c22 = P.C[8 * n + p];
    float dvp = (c00 + c11) + c22;
    float corr = (dvc - dvp) / 3.f;
    P.C[p] = c00 + corr;
    P.C[4 * n + p] = c11 + corr;
    P.C[8 * n + p] = c22 + corr;
}

// ---------------------------------------------------------------------------
// set-up and per-bigStep kernels
// ---------------------------------------------------------------------------
__global__ void k_mu_lam_bulk(int64_t n, const float *E, const float *nu, float *mu, float *lam, float *bulk)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float e = E[p], v = nu[p];
    float m = e / (2.f * (1.f + v));
    float l = (e * v) / ((1.f + v) * (1.f - 2.f * v));
    mu[p] = m; lam[p] = l;
    bulk[p] = l + (2.f / 3.f) * m;
}

__global__ void k_geostatic_F(int64_t n, const float *x, float *F, const float *mu, const float *lam,
                              const float *density, float gravity, float z_top, float K0, int planestrain)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    float depth = z_top - x[2 * n + p];
    float e0, e1, e2;
    if (!planestrain) {
        float sigma_v = (-density[p] * gravity) * depth;
        float sigma_h = K0 * sigma_v;
        float lv = lam[p], mv = mu[p];
        float a11 = 2.f * lv + 2.f * mv, a12 = lv, a21 = 2.f * lv, a22 = lv + 2.f * mv;
        float det = a11 * a22 - a12 * a21;
        float eh = 0.f, ev = 0.f;
        if (fabsf(det) > 1e-12f) {
            eh = (sigma_h * a22 - sigma_v * a12) / det;
            ev = (a11 * sigma_v - a21 * sigma_h) / det;
        }
        e0 = eh; e1 = eh; e2 = ev;
    } else {
        e0 = e1 = e2 = 0.f;
        if (depth > 0.f) {
            float mv = mu[p], lv = lam[p];
            float nu = lv / (2.f * (lv + mv));
            float E = (mv * (3.f * lv + 2.f * mv)) / (lv + mv);
            float sv = (-density[p] * gravity) * depth;
            float sh = K0 * sv;
            float syy = nu * (sh + sv);
            e0 = (sh - nu * (syy + sv)) / E;
            e1 = 0.f;
            e2 = (sv - nu * (sh + syy)) / E;
        }
    }
    float f[9] = {expf(e0), 0.f, 0.f, 0.f, expf(e1), 0.f, 0.f, 0.f, expf(e2)};
    store9(F, n, p, f);
}

__global__ void k_teleport(mpmw_particles_t P, float z_datum, float dist)
{
    const int64_t n = P.n;
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (P.active[p] == 1 && P.material[p] == 2 && P.x[2 * n + p] < z_datum) {
        P.active[p] = 0;
        P.x[2 * n + p] = P.x[2 * n + p] - dist;
        P.v[p] = 0.f; P.v[n + p] = 0.f; P.v[2 * n + p] = 0.f;
    }
}

__global__ void k_creep(mpmw_particles_t P, const float *ys_base, float dt, float base_creep, float damage_creep,
                        float damage_exponent)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P.n) return;
    if (P.material[p] > 1) return;
    float rate = base_creep + damage_creep * powf(P.damage[p], damage_exponent);
    float decay = (rate * ys_base[p]) * dt;
    P.ys[p] = rmax(0.f, P.ys[p] - decay);
}

// Per-step statistics in FP32 and integers (no FP64 arithmetic on the GPU).
// The two sums (|v|/r and damage over active particles) are Kahan-compensated
// per thread, reduced pairwise across the block with the compensation folded
// in, and added across blocks with one FP32 atomic per block (at most 1184
// terms, so the cross-block rounding stays near 1e-7 relative); the five
// counts are exact integer atomics.  While the kernel runs, `out` (7 doubles)
// holds that accumulator (StatsAcc); k_stats_finish converts it in place.
struct StatsAcc {
    float res, dmg;           // sum |v|/r, sum damage over active particles
    unsigned int count[5];    // active, active MPM, active XPBD, inactive MPM, inactive XPBD
};
static_assert(sizeof(StatsAcc) <= 7 * sizeof(double), "the accumulator fits the output");

__device__ __forceinline__ void kahan_add(float &sum, float &c, float x)
{
    const float y = x - c;
    const float t = sum + y;
    c = (t - sum) - y;
    sum = t;
}

__global__ void __launch_bounds__(kBlock) k_stats(mpmw_particles_t P, StatsAcc *acc_out)
{
    const int64_t n = P.n;
    float res = 0.f, res_c = 0.f, dmg = 0.f, dmg_c = 0.f;
    unsigned int cnt[5] = {0u, 0u, 0u, 0u, 0u};
    // every field is loaded whatever the labels, so the loads of several
    // iterations are in flight together
#pragma unroll 4
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const int a = P.active[p], mt = P.material[p];
        float v3[3];
        load3(P.v, n, p, v3);
        const float r = P.radius[p], d = P.damage[p];
        const bool act = a == 1, xp = mt == 2;
        if (act) {
            kahan_add(res, res_c, len3(v3) / r);
            kahan_add(dmg, dmg_c, d);
            ++cnt[0];
        }
        if (xp) { if (act) ++cnt[2]; else ++cnt[4]; }
        else { if (act) ++cnt[1]; else ++cnt[3]; }
    }
    res -= res_c;
    dmg -= dmg_c;
    // pairwise across the warp, then across the warps of the block
    for (int o = 16; o > 0; o >>= 1) {
        res += __shfl_down_sync(0xffffffffu, res, o);
        dmg += __shfl_down_sync(0xffffffffu, dmg, o);
#pragma unroll
        for (int k = 0; k < 5; ++k) cnt[k] += __shfl_down_sync(0xffffffffu, cnt[k], o);
    }
    __shared__ float fr[kBlock / 32], fd[kBlock / 32];
    __shared__ unsigned int fc[5][kBlock / 32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        fr[w] = res; fd[w] = dmg;
#pragma unroll
        for (int k = 0; k < 5; ++k) fc[k][w] = cnt[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.f, b = 0.f;
        unsigned int c[5] = {0u, 0u, 0u, 0u, 0u};
        for (int q = 0; q < kBlock / 32; ++q) {
            a += fr[q]; b += fd[q];
#pragma unroll
            for (int k = 0; k < 5; ++k) c[k] += fc[k][q];
        }
        atomicAdd(&acc_out->res, a);
        atomicAdd(&acc_out->dmg, b);
#pragma unroll
        for (int k = 0; k < 5; ++k)
            if (c[k]) atomicAdd(&acc_out->count[k], c[k]);
    }
}

// the accumulator -> the 7 doubles of mpmw_stats, in place (one thread)
__global__ void k_stats_finish(double *out)
{
    const StatsAcc a = *reinterpret_cast<const StatsAcc *>(out);
    out[0] = (double)a.res;
    out[1] = (double)a.count[0];
    out[2] = (double)a.dmg;
    out[3] = (double)a.count[1];
    out[4] = (double)a.count[2];
    out[5] = (double)a.count[3];
    out[6] = (double)a.count[4];
}

// ---------------------------------------------------------------------------
// argument checks
// ---------------------------------------------------------------------------
// field groups an entry point needs
enum : unsigned { kNeedLabels = 1, kNeedXV = 2, kNeedCF = 4, kNeedStress = 8 };

static int check_particles(const mpmw_particles_t *p, unsigned need)
{
    if (!p) { set_error("particles is NULL"); return MPMW_E_ARG; }
    if (p->n < 0) { set_error("negative particle count"); return MPMW_E_ARG; }
    if (count_too_large(p->n, "particles")) return MPMW_E_ARG;
    if (p->n == 0) return MPMW_OK;
    if ((need & kNeedLabels) && (!p->active || !p->material)) {
        set_error("particles: active and material labels are required");
        return MPMW_E_ARG;
    }
    if ((need & kNeedXV) && (!p->x || !p->v)) { set_error("particles: x and v are required"); return MPMW_E_ARG; }
    if ((need & kNeedCF) && (!p->C || !p->F)) { set_error("particles: C and F are required"); return MPMW_E_ARG; }
    if ((need & kNeedStress) &&
        (!p->F_trial || !p->stress || !p->mu || !p->lam || !p->ys || !p->alpha || !p->hardening || !p->softening ||
         !p->strain_criteria || !p->eta_shear || !p->eta_bulk || !p->acc_strain || !p->damage || !p->density ||
         !p->x_pc || !p->v_pc)) {
        set_error("particles: a stress/material field is NULL");
        return MPMW_E_ARG;
    }
    return MPMW_OK;
}

static int check_grid(const mpmw_grid_t *g)
{
    if (!g) { set_error("grid is NULL"); return MPMW_E_ARG; }
    if (g->dims[0] <= 0 || g->dims[1] <= 0 || g->dims[2] <= 0) { set_error("grid dims must be positive"); return MPMW_E_ARG; }
    if ((int64_t)g->dims[0] * g->dims[1] * g->dims[2] > (int64_t)INT32_MAX) { set_error("grid too large"); return MPMW_E_ARG; }
    if (!g->mv || !g->v) { set_error("grid mv and v are required"); return MPMW_E_ARG; }
    if ((reinterpret_cast<uintptr_t>(g->mv) | reinterpret_cast<uintptr_t>(g->v)) & 15u) {
        set_error("grid mv and v must be 16-byte aligned");
        return MPMW_E_ARG;
    }
    return MPMW_OK;
}

static int check_params(const mpmw_params_t *prm)
{
    if (!prm) { set_error("params is NULL"); return MPMW_E_ARG; }
    if (prm->boundary_condition < -1 || prm->boundary_condition > MPMW_BC_PLANE_STRAIN_Y_GLOBAL) {
        set_error("unknown boundary_condition %d", prm->boundary_condition);
        return MPMW_E_ARG;
    }
    return MPMW_OK;
}

#define MPMW_TRY(expr)            \
    do {                          \
        int _rc = (expr);         \
        if (_rc != MPMW_OK) return _rc; \
    } while (0)

// host-side launchers (also used by the multi-step driver)
// pdl: a programmatic dependent launch (the fused schedule's chain);
// reset: a worklist count the kernel sets to 0
int launch_grid(const mpmw_grid_t &g, const mpmw_params_t &prm, cudaStream_t s, bool zero_mv = false,
                int *reset = nullptr, bool pdl = false)
{
    int64_t G = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (pdl) {
        if (launch_pdl(k_grid_update, grid_for(G), kBlock, 0, s, g, prm, zero_mv ? 1 : 0, reset) != cudaSuccess) {
            set_error("k_grid_update: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            return MPMW_E_DEVICE;
        }
        return MPMW_OK;
    }
    k_grid_update<<<grid_for(G), kBlock, 0, s>>>(g, prm, zero_mv ? 1 : 0, reset);
    return check_launch("k_grid_update");
}
int launch_vlc(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st, cudaStream_t s)
{
    if (!g.cell_div || !g.cell_vol) { set_error("vlc requires grid cell_div and cell_vol"); return MPMW_E_ARG; }
    size_t G = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (cudaMemsetAsync(g.cell_div, 0, G * sizeof(float), s) != cudaSuccess ||
        cudaMemsetAsync(g.cell_vol, 0, G * sizeof(float), s) != cudaSuccess) {
        set_error("vlc: memset failed");
        return MPMW_E_DEVICE;
    }
    if (p.n == 0) return MPMW_OK;
    k_vlc_acc<<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st);
    MPMW_TRY(check_launch("k_vlc_acc"));
    k_vlc_apply<<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st);
    return check_launch("k_vlc_apply");
}
int zero_grid(const mpmw_grid_t &g, cudaStream_t s)
{
    size_t G = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (cudaMemsetAsync(g.mv, 0, G * 4 * sizeof(float), s) != cudaSuccess) {
        set_error("grid memset failed");
        return MPMW_E_DEVICE;
    }
    return MPMW_OK;
}

}  // namespace mpmw

using namespace mpmw;

extern "C" {

const char *mpmw_last_error(void) { return mpmw::g_err; }
int mpmw_version(void) { return 1; }

int mpmw_mu_lam_bulk(int64_t n, const float *E, const float *nu, float *mu, float *lam, float *bulk,
                     mpmw_stream_t stream)
{
    if (n < 0 || (n > 0 && (!E || !nu || !mu || !lam || !bulk))) { set_error("mu_lam_bulk: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "mu_lam_bulk")) return MPMW_E_ARG;
    if (n == 0) return MPMW_OK;
    k_mu_lam_bulk<<<grid_for(n), kBlock, 0, as_stream(stream)>>>(n, E, nu, mu, lam, bulk);
    return check_launch("k_mu_lam_bulk");
}

int mpmw_geostatic_F(int64_t n, const float *x, float *F, const float *mu, const float *lam, const float *density,
                     float gravity, float z_top, float K0, int planestrain, mpmw_stream_t stream)
{
    if (n < 0 || (n > 0 && (!x || !F || !mu || !lam || !density))) { set_error("geostatic_F: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "geostatic_F")) return MPMW_E_ARG;
    if (n == 0) return MPMW_OK;
    k_geostatic_F<<<grid_for(n), kBlock, 0, as_stream(stream)>>>(n, x, F, mu, lam, density, gravity, z_top, K0, planestrain);
    return check_launch("k_geostatic_F");
}

int mpmw_stress(const mpmw_particles_t *p, const mpmw_params_t *prm, uint32_t *status, mpmw_stream_t stream)
{
    (void)status;
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedCF | kNeedStress));
    MPMW_TRY(check_params(prm));
    return launch_stress(*p, *prm, as_stream(stream));
}

int mpmw_p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (p->n > 0 && (!p->stress || !p->vol || !p->mass)) { set_error("p2g: stress, vol and mass are required"); return MPMW_E_ARG; }
    return launch_p2g(*p, *g, *prm, status, as_stream(stream));
}

int mpmw_grid_update(const mpmw_grid_t *g, const mpmw_params_t *prm, mpmw_stream_t stream)
{
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    return launch_grid(*g, *prm, as_stream(stream));
}

int mpmw_grid_op(const mpmw_grid_t *g, const mpmw_params_t *prm, int op, mpmw_stream_t stream)
{
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (op < 0 || op > 2) { set_error("grid_op: unknown op %d", op); return MPMW_E_ARG; }
    if (op == 2 && prm->boundary_condition < 0) return MPMW_OK;
    int64_t G = (int64_t)g->dims[0] * g->dims[1] * g->dims[2];
    k_grid_op<<<grid_for(G), kBlock, 0, as_stream(stream)>>>(*g, *prm, op);
    return check_launch("k_grid_op");
}

int mpmw_g2p(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (p->n > 0 && !p->F_trial) { set_error("g2p: F_trial is required"); return MPMW_E_ARG; }
    if (prm->update_cov && p->n > 0 && !p->cov) { set_error("g2p: update_cov needs cov"); return MPMW_E_ARG; }
    return launch_g2p(*p, *g, *prm, status, false, nullptr, 0, as_stream(stream));
}

size_t mpmw_workspace_bytes(int64_t n) { return mpmw::g2p_workspace_bytes(n < 0 ? 0 : n); }

int mpmw_g2p_stress(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
                    void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (prm->update_cov && p->n > 0 && !p->cov) { set_error("g2p: update_cov needs cov"); return MPMW_E_ARG; }
    return launch_g2p(*p, *g, *prm, status, true, workspace, ws_bytes, as_stream(stream));
}

int mpmw_stress_p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
                    void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (p->n > 0 && (!p->vol || !p->mass)) { set_error("stress_p2g: vol and mass are required"); return MPMW_E_ARG; }
    return launch_stress_p2g(*p, *g, *prm, status, workspace, ws_bytes, as_stream(stream));
}

int mpmw_g2p2g(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int store_stress,
               uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (p->n > 0 && (!p->vol || !p->mass)) { set_error("g2p2g: vol and mass are required"); return MPMW_E_ARG; }
    if (prm->update_cov && p->n > 0 && !p->cov) { set_error("g2p2g: update_cov needs cov"); return MPMW_E_ARG; }
    return launch_g2p2g(*p, *g, *prm, status, store_stress != 0, workspace, ws_bytes, as_stream(stream));
}

int mpmw_vlc(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
             mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (p->n > 0 && !p->vol) { set_error("vlc: vol is required"); return MPMW_E_ARG; }
    return launch_vlc(*p, *g, *prm, status, as_stream(stream));
}

int mpmw_vlc_phase(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int phase,
                   uint32_t *status, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels));
    MPMW_TRY(check_params(prm));
    if (!g || g->dims[0] <= 0 || g->dims[1] <= 0 || g->dims[2] <= 0 || !g->cell_div || !g->cell_vol) {
        set_error("vlc_phase: grid dims and cell_div/cell_vol are required");
        return MPMW_E_ARG;
    }
    if (phase != 0 && phase != 1) { set_error("vlc_phase: phase must be 0 or 1"); return MPMW_E_ARG; }
    if (p->n == 0) return MPMW_OK;
    if (!p->x || !p->C || (phase == 0 && !p->vol)) { set_error("vlc_phase: x, C (and vol) are required"); return MPMW_E_ARG; }
    cudaStream_t s = as_stream(stream);
    if (phase == 0) k_vlc_acc<<<grid_for(p->n), kBlock, 0, s>>>(*p, *g, *prm, status);
    else k_vlc_apply<<<grid_for(p->n), kBlock, 0, s>>>(*p, *g, *prm, status);
    return check_launch(phase == 0 ? "k_vlc_acc" : "k_vlc_apply");
}

int mpmw_substep(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, uint32_t *status,
                 mpmw_stream_t stream)
{
    return mpmw_run_substeps(p, g, prm, 1, status, nullptr, 0, stream);
}

int mpmw_run_substeps(const mpmw_particles_t *p, const mpmw_grid_t *g, const mpmw_params_t *prm, int nsteps,
                      uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    MPMW_TRY(check_grid(g));
    MPMW_TRY(check_params(prm));
    if (nsteps < 0) { set_error("nsteps must be >= 0"); return MPMW_E_ARG; }
    if (p->n > 0 && (!p->vol || !p->mass)) { set_error("substep: vol and mass are required"); return MPMW_E_ARG; }
    if (prm->update_cov && p->n > 0 && !p->cov) { set_error("substep: update_cov needs cov"); return MPMW_E_ARG; }
    if (prm->vlc && (!g->cell_div || !g->cell_vol)) { set_error("substep: vlc needs cell_div/cell_vol"); return MPMW_E_ARG; }
    cudaStream_t s = as_stream(stream);
    if (nsteps == 0) return MPMW_OK;
    // Fused schedule (no VLC, workspace given): after the first substep's
    // stress + P2G, each grid update also clears the accumulators and one
    // G2P->P2G kernel carries substep k's G2P, substep k+1's return map and
    // substep k+1's P2G; the last substep ends with the plain G2P.  Otherwise
    // every substep is stress, P2G, grid update, G2P (+ VLC).  With a
    // workspace, each stress + P2G is one kernel (k_stress_p2g).
    const bool fuse = !prm->vlc && workspace != nullptr;
    auto stress_then_p2g = [&]() -> int {
        MPMW_TRY(zero_grid(*g, s));
        if (workspace) return launch_stress_p2g(*p, *g, *prm, status, workspace, ws_bytes, s);
        MPMW_TRY(launch_stress(*p, *prm, s));
        return launch_p2g(*p, *g, *prm, status, s);
    };
    MPMW_TRY(stress_then_p2g());
    for (int step = 0; step < nsteps; ++step) {
        const bool last = step == nsteps - 1;
        if (!last && fuse) {
            // grid update -> fused kernel -> worklist as one chain of
            // programmatic dependent launches: each kernel's CTAs are
            // scheduled during its predecessor's last wave and wait for it to
            // finish, which hides the launch gaps.  The grid pass also resets
            // the fused kernel's worklist count.
            MPMW_TRY(launch_grid(*g, *prm, s, true, static_cast<int *>(workspace), true));
            MPMW_TRY(launch_g2p2g(*p, *g, *prm, status, step + 1 == nsteps - 1, workspace, ws_bytes, s, true));
        } else {
            MPMW_TRY(launch_grid(*g, *prm, s));
            MPMW_TRY(launch_g2p(*p, *g, *prm, status, false, nullptr, 0, s));
            if (prm->vlc) MPMW_TRY(launch_vlc(*p, *g, *prm, status, s));
            if (!last) MPMW_TRY(stress_then_p2g());
        }
    }
    return MPMW_OK;
}

size_t mpmw_batch_workspace_bytes(const mpmw_grid_t *grids, int nscenes, int64_t n)
{
    if (!grids || nscenes < 1 || n < 0) return 0;
    for (int k = 0; k < nscenes; ++k)
        if (grids[k].dims[0] <= 0 || grids[k].dims[1] <= 0 || grids[k].dims[2] <= 0) return 0;
    return batch_workspace_bytes(grids, nscenes, n);
}

int mpmw_batch_prepare(const mpmw_particles_t *p, const mpmw_grid_t *grids, const mpmw_params_t *prms,
                       const int64_t *offsets, int nscenes, void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    if (!grids || !prms || !offsets) { set_error("batch: grids, prms and offsets are required"); return MPMW_E_ARG; }
    if (nscenes < 1) { set_error("batch: %d scenes (at least 1)", nscenes); return MPMW_E_ARG; }
    if (p->n > 0 && (!p->vol || !p->mass)) { set_error("batch: vol and mass are required"); return MPMW_E_ARG; }
    if (offsets[0] != 0 || offsets[nscenes] != p->n) {
        set_error("batch: offsets must run from 0 to the particle count %lld", (long long)p->n);
        return MPMW_E_ARG;
    }
    for (int k = 0; k < nscenes; ++k) {
        MPMW_TRY(check_grid(&grids[k]));
        MPMW_TRY(check_params(&prms[k]));
        if (offsets[k + 1] <= offsets[k] || offsets[k] % 256 != 0) {
            set_error("batch: scene %d: offsets must increase and be multiples of 256", k);
            return MPMW_E_ARG;
        }
        if (prms[k].vlc) { set_error("batch: scene %d: volumetric locking correction is not batched", k); return MPMW_E_ARG; }
        if (prms[k].update_cov && !p->cov) { set_error("batch: scene %d: update_cov needs cov", k); return MPMW_E_ARG; }
    }
    if (!workspace) { set_error("batch: workspace is NULL"); return MPMW_E_WORKSPACE; }
    return prepare_batch(*p, grids, prms, offsets, nscenes, workspace, ws_bytes, as_stream(stream));
}

int mpmw_batch_run_substeps(const mpmw_particles_t *p, int nsteps, uint32_t *status, void *workspace,
                            size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    if (nsteps < 0) { set_error("nsteps must be >= 0"); return MPMW_E_ARG; }
    if (!workspace) { set_error("batch: workspace is NULL"); return MPMW_E_WORKSPACE; }
    return launch_batch_substeps(*p, 0, -1, nsteps, status, workspace, ws_bytes, as_stream(stream));
}

int mpmw_batch_run_range(const mpmw_particles_t *p, int first_scene, int last_scene, int nsteps, uint32_t *status,
                         void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    if (nsteps < 0) { set_error("nsteps must be >= 0"); return MPMW_E_ARG; }
    if (!workspace) { set_error("batch: workspace is NULL"); return MPMW_E_WORKSPACE; }
    return launch_batch_substeps(*p, first_scene, last_scene, nsteps, status, workspace, ws_bytes,
                                 as_stream(stream));
}

int mpmw_batch_run_persistent(const mpmw_particles_t *p, int nsteps, uint32_t *status, void *workspace,
                              size_t ws_bytes, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV | kNeedCF | kNeedStress));
    if (nsteps < 0) { set_error("nsteps must be >= 0"); return MPMW_E_ARG; }
    if (!workspace) { set_error("batch: workspace is NULL"); return MPMW_E_WORKSPACE; }
    return launch_batch_persistent(*p, nsteps, status, workspace, ws_bytes, as_stream(stream));
}

int64_t mpmw_batch_persistent_launches(void) { return batch_persistent_launches(); }

int mpmw_batch_set_options(const void *workspace, int gather_tile, int read_ahead)
{
    if (!workspace) { set_error("batch: workspace is NULL"); return MPMW_E_ARG; }
    if (!set_batch_options(workspace, gather_tile, read_ahead)) {
        set_error("batch: the workspace was not prepared (mpmw_batch_prepare)");
        return MPMW_E_ARG;
    }
    return MPMW_OK;
}

int mpmw_teleport(const mpmw_particles_t *p, float z_datum, float teleport_distance, mpmw_stream_t stream)
{
    MPMW_TRY(check_particles(p, kNeedLabels | kNeedXV));
    if (p->n == 0) return MPMW_OK;
    k_teleport<<<grid_for(p->n), kBlock, 0, as_stream(stream)>>>(*p, z_datum, teleport_distance);
    return check_launch("k_teleport");
}

int mpmw_creep(const mpmw_particles_t *p, const float *ys_base, float dt, float base_creep, float damage_creep,
               float damage_exponent, mpmw_stream_t stream)
{
    if (!p || p->n < 0 || (p->n > 0 && (!p->material || !p->damage || !p->ys || !ys_base))) {
        set_error("creep: bad arguments");
        return MPMW_E_ARG;
    }
    if (count_too_large(p->n, "creep")) return MPMW_E_ARG;
    if (p->n == 0) return MPMW_OK;
    k_creep<<<grid_for(p->n), kBlock, 0, as_stream(stream)>>>(*p, ys_base, dt, base_creep, damage_creep, damage_exponent);
    return check_launch("k_creep");
}

int mpmw_stats(const mpmw_particles_t *p, double *out, mpmw_stream_t stream)
{
    if (!p || p->n < 0 || !out) { set_error("stats: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(p->n, "stats")) return MPMW_E_ARG;
    if (p->n > 0 && (!p->active || !p->material || !p->v || !p->radius || !p->damage)) {
        set_error("stats: active, material, v, radius and damage are required");
        return MPMW_E_ARG;
    }
    if ((reinterpret_cast<uintptr_t>(out) & 7u) != 0) { set_error("stats: out must be 8-byte aligned"); return MPMW_E_ARG; }
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(out, 0, 7 * sizeof(double), s) != cudaSuccess) { set_error("stats: memset failed"); return MPMW_E_DEVICE; }
    if (p->n == 0) return MPMW_OK;
    int64_t blocks = (p->n + kBlock - 1) / kBlock;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_stats<<<(unsigned)blocks, kBlock, 0, s>>>(*p, reinterpret_cast<StatsAcc *>(out));
    MPMW_TRY_LAUNCH("k_stats");
    k_stats_finish<<<1, 1, 0, s>>>(out);
    return check_launch("k_stats_finish");
}

}  // extern "C"
