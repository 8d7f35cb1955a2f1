// mpmw_g2p.cu -- grid-to-particle transfer (reference: utils/mpmRoutines.py:715-802
// g2p + update_cov), the stress kernels (:229-312) and the fused substep kernel.
//
// k_g2p<false>: the reference's g2p (x, v, C, F_trial).
// k_g2p<true>:  g2p followed, in registers, by the next substep's return map in
//   tensor form (mpmw_stress.cuh).  Particles that need the SVD path (large
//   deformation, reflection, or stress_mode SVD) get their F_trial written and
//   their index appended to a worklist that k_stress_list finishes.
// k_g2p2g:      g2p, the next substep's return map and that substep's P2G
//   (mpmw_scatter.cuh) in one pass.  v, C and the stress stay in registers from
//   the gather to the scatter: per substep the kernel reads x, labels, F, the
//   material scalars, mass and volume and writes x and F (the stress too on the
//   last fused step; v and C are rewritten by the final, unfused G2P of a run).
//   SVD-path particles are listed; k_stress_p2g_list finishes their return map
//   and scatters them with global atomics.
// k_stress_p2g: a substep's return map (from F_trial) and its P2G in one pass,
//   the first half of a substep whenever a workspace is given; SVD-path
//   particles go to the same worklist and k_stress_p2g_list.
// The worklists live in the caller's workspace (mpmw_workspace_bytes).
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "mpmw_common.cuh"
#include "mpmw_gather.cuh"
#include "mpmw_gridsync.cuh"
#include "mpmw_grid.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"
#include "mpmw_scatter.cuh"
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

// SVD-path stress + P2G scatter of one particle listed by k_g2p2g
__device__ __forceinline__ void stress_p2g_one(const mpmw_particles_t &P, const mpmw_grid_t &G,
                                               const mpmw_params_t &prm, int64_t p, uint32_t &bad)
{
    const int64_t n = P.n;
    float Ft[9], Cg[9], Fo[9], out[9];
    load9(P.F_trial, n, p, Ft);
    load9(P.C, n, p, Cg);
    stress_particle<false>(P, prm.eff, MPMW_STRESS_SVD, p, Ft, Cg, nullptr, nullptr, Fo, out);
    store9(P.F, n, p, Fo);
    store_sym6(P.stress, n, p, out);
    if (P.material[p] <= 1) {
        float xp[3], v[3];
        load3(P.x, n, p, xp);
        load3(P.v, n, p, v);
        const float st6[6] = {out[0], out[4], out[8], out[1], out[2], out[5]};
        p2g_scatter_one(xp, v, Cg, st6, P.mass[p], P.vol[p], prm, reinterpret_cast<float4 *>(G.mv), G.dims[0],
                        G.dims[1], G.dims[2], bad);
    }
}

// SVD-path stress + P2G scatter for the particles listed by k_g2p2g
__global__ void __launch_bounds__(kBlock) k_stress_p2g_list(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                           uint32_t *status, const int *__restrict__ list,
                                                           const int *__restrict__ count)
{
    pdl_wait();
    pdl_trigger();
    const int cnt = *count;
    uint32_t bad = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x)
        stress_p2g_one(P, G, prm, list[q], bad);
    if (bad) raise_status(status, bad);
}

// Shared memory of k_g2p: the grid tile, F of the CTA's particles (read ahead
// by bulk copies) and the positions, parked while the gather runs so that fewer
// registers stay live across it.
template <int Cta>
struct G2PShared {
    GatherShared g;
    float F[9][Cta];
    float xpark[3][Cta];
    uint64_t pbar;
};

// G2P of the CTA of Cta particles (and threads) that starts at p0 (a multiple
// of Cta).
template <bool Fused, int Cta = kBlock>
__device__ __forceinline__ void g2p_body(const mpmw_particles_t &P, const mpmw_grid_t &G, const mpmw_params_t &prm,
                                         uint32_t *status, int *svd_list, int *svd_count, const CUtensorMap *tmap,
                                         int use_tma, int use_ahead, int64_t p0)
{
    static_assert(Cta % 32 == 0 && Cta / 32 <= kGatherMaxWarps, "whole warps, within the gather's box slots");
    __shared__ __align__(128) G2PShared<Cta> S;
    const int64_t n = P.n;
    const int t = threadIdx.x;
    const int64_t p = p0 + t;
    // F read ahead into shared memory by bulk copies (full CTAs; the host checks
    // the 16-byte alignment they need), in flight while the CTA waits for its tile
    const bool ahead = use_ahead && p0 + Cta <= n;
    if (ahead && t == 0) {
        mbar_init(&S.pbar, 1);
        mbar_arrive_expect_tx(&S.pbar, 9u * Cta * 4u);
#pragma unroll 1
        for (int f = 0; f < 9; ++f) bulk_load(&S.F[f][0], P.F + (int64_t)f * n + p0, Cta * 4u, &S.pbar);
    }
    // labels and x are loaded together (not behind the label test)
    int lab_a = 0, lab_m = 0;
    float xp[3] = {0.f, 0.f, 0.f};
    if (p < n) {
        lab_a = P.active[p];
        lab_m = P.material[p];
        load3(P.x, n, p, xp);
    }
    const bool act = lab_a == 1 && lab_m <= 1;
    Weights W;
    if (act) weights(xp, prm.min_bounds, prm.inv_dx, W);
#pragma unroll
    for (int a = 0; a < 3; ++a) S.xpark[a][t] = xp[a];
    bool tile = false;
    int ox = 0, oy = 0, oz = 0;
    if (!gather_prepare(S.g, act, W, tmap, use_tma, status, tile, ox, oy, oz)) {
        // no active particle: the read-ahead must still land before the CTA exits
        if (ahead && !mbar_wait_bounded(&S.pbar, 0)) raise_status(status, MPMW_ST_TIMEOUT);
        return;  // uniform
    }
    // every active thread waits for the read-ahead, so the CTA outlives the copies
    if (!act) return;
    uint32_t bad = 0;
    float nv[3], nF[9], nC[9];
    gather_particle(S.g, tile, ox, oy, oz, W, G, prm.inv_dx, nv, nF, nC, bad);
    float xn[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) xn[a] = fma_(prm.dt, nv[a], S.xpark[a][t]);
    if (!(isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]))) bad |= MPMW_ST_NAN;
    float Fpre[9];
    bool ahead_ok = ahead;
    if (ahead && !mbar_wait_bounded(&S.pbar, 0)) {
        // report, wait once more for the copies in flight, and read global memory
        bad |= MPMW_ST_TIMEOUT;
        mbar_wait_bounded(&S.pbar, 0);
        ahead_ok = false;
    }
    if (ahead_ok) {
#pragma unroll
        for (int k = 0; k < 9; ++k) Fpre[k] = S.F[k][t];
    } else {
        load9(P.F, n, p, Fpre);
    }
    float Ft[9];
    g2p_deformation(P, prm, p, nF, Ft, Fpre);
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

template <bool Fused>
__global__ void __launch_bounds__(kBlock, 3) k_g2p(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                               uint32_t *status, int *svd_list, int *svd_count,
                                               const __grid_constant__ CUtensorMap tmap, int use_tma, int use_ahead)
{
    g2p_body<Fused>(P, G, prm, status, svd_list, svd_count, &tmap, use_tma, use_ahead,
                    (int64_t)blockIdx.x * blockDim.x);
}

struct G2P2GShared {
    GatherShared g;
    ScatterShared s;
    uint64_t pbar;  // particle-field read-ahead
};

// Particle fields the fused body can read ahead (bulk copies into the
// scatter's record area, which is free until the scatter) when its caller asks
// for it -- the batched kernels' tuner option; the single-scene launch loads
// them plainly: F (9), mu, lam, ys, alpha, damage, eta_shear, eta_bulk, mass,
// vol.
constexpr int kAheadFields = 18;
struct AheadFields {
    float f[kAheadFields][kScatterChunk];
};
static_assert(sizeof(AheadFields) <= sizeof(ScatterShared::rec), "read-ahead fits the record area");
// the particle positions are parked in the record area behind the read-ahead
// fields while the gather runs (fewer registers live across it)
static_assert((kAheadFields + 3) * kScatterChunk * sizeof(float) <= sizeof(ScatterShared::rec),
              "parked positions fit the record area");

__device__ __forceinline__ const float *ahead_src(const mpmw_particles_t &P, int field)
{
    const int64_t n = P.n;
    if (field < 9) return P.F + (int64_t)field * n;
    switch (field) {
    case 9: return P.mu;
    case 10: return P.lam;
    case 11: return P.ys;
    case 12: return P.alpha;
    case 13: return P.damage;
    case 14: return P.eta_shear;
    case 15: return P.eta_bulk;
    case 16: return P.mass;
    default: return P.vol;
    }
}

// G2P of substep k, return map of substep k+1, P2G of substep k+1 (into grid.mv,
// which the caller has zeroed) for the CTA whose particles start at p0 (a
// multiple of kScatterChunk).  StoreStress: also write the stress (the last
// fused substep of a run).
template <bool StoreStress>
__device__ __forceinline__ void g2p2g_body(const mpmw_particles_t &P, const mpmw_grid_t &G, const mpmw_params_t &prm,
                                           uint32_t *status, int *svd_list, int *svd_count, const CUtensorMap *tmap,
                                           int use_tma, int use_ahead, int64_t p0, bool store_rt = false)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // the TMA destination (S.g.tile) must be 128-byte aligned: round the base up
    // (the launch reserves 128 bytes for this)
    G2P2GShared &S = *reinterpret_cast<G2P2GShared *>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    const int64_t n = P.n;
    const int t = threadIdx.x;
    const int64_t p = p0 + t;
    // optional read-ahead of the particle fields used after the gather (full
    // CTAs only; the host checks the 16-byte alignment the bulk copies need)
    const bool ahead = use_ahead && p0 + kScatterChunk <= n;
    AheadFields &AF = *reinterpret_cast<AheadFields *>(&S.s.rec[0][0]);
    if (ahead && t == 0) {
        mbar_init(&S.pbar, 1);
        mbar_arrive_expect_tx(&S.pbar, kAheadFields * kScatterChunk * 4u);
#pragma unroll 1
        for (int f = 0; f < kAheadFields; ++f) bulk_load(&AF.f[f][0], ahead_src(P, f) + p0, kScatterChunk * 4u, &S.pbar);
    }
    // the scatter's counting-sort bins and out-of-box flag, cleared here and
    // published by the gather's first barrier (the scatter then needs no box
    // reduction of its own: see below)
    for (int q = t; q < kScatterBins; q += kScatterChunk) S.s.bins[q] = 0;
    if (t == 0) S.s.outside = 0;
    // labels and x are loaded together (not behind the label test)
    int lab_a = 0, lab_m = 0;
    float xp[3] = {0.f, 0.f, 0.f};
    if (p < n) {
        lab_a = P.active[p];
        lab_m = P.material[p];
        load3(P.x, n, p, xp);
    }
    const bool act = lab_a == 1 && lab_m <= 1;
    Weights W;
    if (act) weights(xp, prm.min_bounds, prm.inv_dx, W);
    float(*xpark)[kScatterChunk] = &AF.f[0] + kAheadFields;
#pragma unroll
    for (int a = 0; a < 3; ++a) xpark[a][t] = xp[a];
    bool tile = false;
    int ox = 0, oy = 0, oz = 0;
    if (!gather_prepare(S.g, act, W, tmap, use_tma, status, tile, ox, oy, oz)) {
        // no active particle: the read-ahead must still land before the CTA exits
        if (ahead && !mbar_wait_bounded(&S.pbar, 0)) raise_status(status, MPMW_ST_TIMEOUT);
        return;  // uniform
    }
    uint32_t bad = 0;
    bool ahead_ok = ahead;
    if (ahead && !mbar_wait_bounded(&S.pbar, 0)) {
        // report, wait once more for the copies in flight, and read global memory
        raise_status(status, MPMW_ST_TIMEOUT);
        mbar_wait_bounded(&S.pbar, 0);
        ahead_ok = false;
    }

    bool scat = false;
    float xn[3] = {0.f, 0.f, 0.f}, nv[3] = {0.f, 0.f, 0.f}, nC[9], st6[6];
    float m = 0.f, vol = 0.f;
    if (act) {
        float nF[9];
        gather_particle(S.g, tile, ox, oy, oz, W, G, prm.inv_dx, nv, nF, nC, bad);
#pragma unroll
        for (int a = 0; a < 3; ++a) xn[a] = fma_(prm.dt, nv[a], xpark[a][t]);
        if (!(isfinite(xn[0]) && isfinite(xn[1]) && isfinite(xn[2]))) bad |= MPMW_ST_NAN;
        float Ft[9];
        {
            float Fpre[9];
            if (ahead_ok) {
#pragma unroll
                for (int k = 0; k < 9; ++k) Fpre[k] = AF.f[k][t];
            } else {
                load9(P.F, n, p, Fpre);
            }
            g2p_deformation(P, prm, p, nF, Ft, Fpre);
        }
        store3(P.x, n, p, xn);
        MatScalars ms;
        float eta_s, eta_b;
        if (ahead_ok) {
            ms.mu = AF.f[9][t]; ms.lam = AF.f[10][t]; ms.ys = AF.f[11][t]; ms.alpha = AF.f[12][t]; ms.D = AF.f[13][t];
            eta_s = AF.f[14][t]; eta_b = AF.f[15][t]; m = AF.f[16][t]; vol = AF.f[17][t];
        } else {
            ms.mu = P.mu[p]; ms.lam = P.lam[p]; ms.ys = P.ys[p]; ms.alpha = P.alpha[p]; ms.D = P.damage[p];
            eta_s = P.eta_shear[p]; eta_b = P.eta_bulk[p]; m = P.mass[p]; vol = P.vol[p];
        }
        float Fo[9], T[9];
        const int rm = prm.stress_mode == MPMW_STRESS_AUTO
                           ? small_strain_update<true>(P, prm.eff, p, Ft, xn, nv, Fo, T, &ms)
                           : 0;
        if (rm != 0) {
            float out[9];
            add_viscous(T, nC, eta_s, eta_b, out);
            store9(P.F, n, p, Fo);
            st6[0] = out[0]; st6[1] = out[4]; st6[2] = out[8]; st6[3] = out[1]; st6[4] = out[2]; st6[5] = out[5];
            if (StoreStress || store_rt || rm == 2) store_sym6(P.stress, n, p, out);
            if (rm == 2) {
                // became an XPBD particle: it leaves the MPM path with this G2P's v and C
                store3(P.v, n, p, nv);
                store9(P.C, n, p, nC);
            } else {
                scat = true;
            }
        } else {
            store9(P.F_trial, n, p, Ft);
            store3(P.v, n, p, nv);
            store9(P.C, n, p, nC);
            svd_list[atomicAdd(svd_count, 1)] = (int)p;
        }
    }
    // A particle moves less than a cell per substep, so the gather's box of
    // stencil bases (old positions), one cell wider on each side, holds every
    // new base; a particle outside it sends the CTA to the scatter's
    // compaction path.
    ScatterBox box;
    bool have_box = true;
    int64_t cells = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int64_t lo = (int64_t)S.g.lo[a] - 1, e = (int64_t)S.g.hi[a] - S.g.lo[a] + 3;
        have_box = have_box && e > 0 && e <= kScatterBins && lo >= INT32_MIN;
        box.lo[a] = have_box ? (int)lo : 0;
        box.ext[a] = have_box ? (int)e : 1;
        cells *= have_box ? e : 1;
    }
    have_box = have_box && cells <= kScatterBins;
    p2g_scatter(S.s, scat, xn, nv, nC, st6, m, vol, prm, reinterpret_cast<float4 *>(G.mv), G.dims[0], G.dims[1],
                G.dims[2], bad, have_box ? &box : nullptr);
    if (bad) raise_status(status, bad);
}

template <bool StoreStress>
__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_g2p2g(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                        uint32_t *status, int *svd_list, int *svd_count,
                                                        const __grid_constant__ CUtensorMap tmap, int use_tma,
                                                        int use_ahead)
{
    pdl_wait();
    pdl_trigger();
    g2p2g_body<StoreStress>(P, G, prm, status, svd_list, svd_count, &tmap, use_tma, use_ahead,
                            (int64_t)blockIdx.x * blockDim.x);
}

// The return map of a substep and its P2G in one pass (the reference's
// compute_stress_from_F_trial followed by p2g_apic_with_stress): F_trial -> F
// and stress (tensor form, in registers) and the CTA-cooperative scatter.  The
// stress is written as the unfused stress kernel writes it; particles that
// need the SVD path are listed for k_stress_p2g_list, particles that become
// XPBD particles write their new v and do not scatter.
// (for the CTA whose particles start at p0, a multiple of kScatterChunk)
__device__ __forceinline__ void stress_p2g_body(const mpmw_particles_t &P, const mpmw_grid_t &G,
                                                const mpmw_params_t &prm, uint32_t *status, int *svd_list,
                                                int *svd_count, int64_t p0)
{
    extern __shared__ __align__(16) unsigned char smem_sp[];
    ScatterShared &S = *reinterpret_cast<ScatterShared *>(smem_sp);
    const int64_t n = P.n;
    const int64_t p = p0 + threadIdx.x;
    bool scat = false;
    float xp[3] = {0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f}, Cg[9], st6[6], Ft[9];
    float m = 0.f, vol = 0.f;
    uint32_t bad = 0;
    // labels and every field the elastic path reads are loaded together (not
    // behind the label test, not inside the return map)
    int lab_a = 0, lab_m = 0;
    MatScalars ms{0.f, 0.f, 0.f, 0.f, 0.f};
    float eta_s = 0.f, eta_b = 0.f, mass = 0.f, volume = 0.f;
    if (p < n) {
        lab_a = P.active[p];
        lab_m = P.material[p];
        load9(P.F_trial, n, p, Ft);
        load9(P.C, n, p, Cg);
        load3(P.x, n, p, xp);
        load3(P.v, n, p, v);
        ms.mu = P.mu[p]; ms.lam = P.lam[p]; ms.ys = P.ys[p]; ms.alpha = P.alpha[p]; ms.D = P.damage[p];
        eta_s = P.eta_shear[p]; eta_b = P.eta_bulk[p];
        mass = P.mass[p]; volume = P.vol[p];
    }
    const bool act = lab_a == 1 && lab_m <= 1;
    if (act) {
        float Fo[9], T[9];
        const int rm = prm.stress_mode == MPMW_STRESS_AUTO
                           ? small_strain_update<true>(P, prm.eff, p, Ft, xp, v, Fo, T, &ms)
                           : 0;
        if (rm != 0) {
            float out[9];
            add_viscous(T, Cg, eta_s, eta_b, out);
            store9(P.F, n, p, Fo);
            store_sym6(P.stress, n, p, out);
            if (rm == 2) {
                store3(P.v, n, p, v);  // became an XPBD particle: its v changed, it does not scatter
            } else {
                st6[0] = out[0]; st6[1] = out[4]; st6[2] = out[8]; st6[3] = out[1]; st6[4] = out[2]; st6[5] = out[5];
                m = mass;
                vol = volume;
                scat = true;
            }
        } else {
            const int slot = atomicAdd(svd_count, 1);
            svd_list[slot] = (int)p;
        }
    }
    p2g_scatter(S, scat, xp, v, Cg, st6, m, vol, prm, reinterpret_cast<float4 *>(G.mv), G.dims[0], G.dims[1],
                G.dims[2], bad);
    if (bad) raise_status(status, bad);
}

__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_stress_p2g(mpmw_particles_t P, mpmw_grid_t G, mpmw_params_t prm,
                                                             uint32_t *status, int *svd_list, int *svd_count)
{
    stress_p2g_body(P, G, prm, status, svd_list, svd_count, (int64_t)blockIdx.x * kScatterChunk);
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
    if (g_maps.size() > 512) g_maps.clear();
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
    // the F read-ahead needs each row's chunk start 16-byte aligned
    const int use_ahead = p.F && p.n % 4 == 0 && (reinterpret_cast<uintptr_t>(p.F) & 15u) == 0 ? 1 : 0;
    if (!fused) {
        k_g2p<false><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st, nullptr, nullptr, map, use_tma, use_ahead);
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
    k_g2p<true><<<grid_for(p.n), kBlock, 0, s>>>(p, g, prm, st, list, count, map, use_tma, use_ahead);
    MPMW_TRY_LAUNCH("k_g2p<fused>");
    k_stress_list<<<148 * 4, kBlock, 0, s>>>(p, prm.eff, list, count);
    return check_launch("k_stress_list");
}

static bool g_g2p2g_attr[64];
static bool g_stress_p2g_attr[64];

// Opts the fused kernels into their shared memory (once per device).  Also
// called before a graph capture, so that no attribute call runs inside one.
int reserve_fused_smem()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_error("no current device"); return MPMW_E_DEVICE; }
    if (dev < 0 || dev >= 64) return MPMW_OK;
    if (!g_g2p2g_attr[dev]) {
        const int smem = (int)(sizeof(G2P2GShared) + 128);
        if (cudaFuncSetAttribute(k_g2p2g<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_g2p2g<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
            set_error("g2p2g: cannot reserve %d bytes of shared memory", smem);
            return MPMW_E_DEVICE;
        }
        g_g2p2g_attr[dev] = true;
    }
    if (!g_stress_p2g_attr[dev]) {
        const int smem = (int)sizeof(ScatterShared);
        if (cudaFuncSetAttribute(k_stress_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) {
            set_error("stress_p2g: cannot reserve %d bytes of shared memory", smem);
            return MPMW_E_DEVICE;
        }
        g_stress_p2g_attr[dev] = true;
    }
    return MPMW_OK;
}

// the read-ahead bulk copies of k_g2p2g need every field's chunk start 16-byte aligned
static bool g2p2g_ahead_ok(const mpmw_particles_t &p)
{
    if (p.n % 4 != 0) return false;
    for (int f = 0; f < kAheadFields; ++f) {
        const float *base = f < 9 ? p.F + (int64_t)f * p.n
                                  : (f == 9 ? p.mu : f == 10 ? p.lam : f == 11 ? p.ys : f == 12 ? p.alpha
                                     : f == 13 ? p.damage : f == 14 ? p.eta_shear : f == 15 ? p.eta_bulk
                                     : f == 16 ? p.mass : p.vol);
        if (!base || (reinterpret_cast<uintptr_t>(base) & 15u) != 0) return false;
    }
    return true;
}

constexpr bool kFusedReadAhead = false;

int launch_g2p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st,
                 bool store_stress, void *ws, size_t ws_bytes, cudaStream_t s, bool chained)
{
    if (p.n == 0) return MPMW_OK;
    if (!ws || ws_bytes < g2p_workspace_bytes(p.n)) {
        set_error("run_substeps: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  g2p_workspace_bytes(p.n));
        return MPMW_E_WORKSPACE;
    }
    const size_t smem = sizeof(G2P2GShared) + 128;  // + alignment slack (see k_g2p2g)
    if (const int rc_ = reserve_fused_smem()) return rc_;
    CUtensorMap map;
    int use_tma = cached_grid_map(g, &map) ? 1 : 0;
    if (!use_tma) memset(&map, 0, sizeof(map));
    int *count = static_cast<int *>(ws);
    int *list = reinterpret_cast<int *>(static_cast<char *>(ws) + 256);
    if (!chained && cudaMemsetAsync(count, 0, sizeof(int), s) != cudaSuccess) {
        set_error("g2p2g: memset failed");
        return MPMW_E_DEVICE;
    }
    // The bulk read-ahead of the particle fields is off here: with 128-particle
    // CTAs its 18 copies of 512 B per CTA cost more than the plain loads (the
    // fused launch on the 3.87 M-particle tunnel: 0.5277 ms without, 0.5372 ms
    // with; an L2 prefetch of the fields at the CTA's start was slower still).
    // The batched kernels keep it as an option their tuner measures.
    const int use_ahead = kFusedReadAhead && g2p2g_ahead_ok(p) ? 1 : 0;
    const unsigned grid = grid_for(p.n, kScatterChunk);
    if (chained) {
        const cudaError_t e = store_stress
            ? launch_pdl(k_g2p2g<true>, grid, kScatterChunk, smem, s, p, g, prm, st, list, count, map, use_tma, use_ahead)
            : launch_pdl(k_g2p2g<false>, grid, kScatterChunk, smem, s, p, g, prm, st, list, count, map, use_tma, use_ahead);
        if (e != cudaSuccess ||
            launch_pdl(k_stress_p2g_list, 148 * 4, kBlock, 0, s, p, g, prm, st, list, (const int *)count) != cudaSuccess) {
            set_error("g2p2g: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            return MPMW_E_DEVICE;
        }
        return MPMW_OK;
    }
    if (store_stress) k_g2p2g<true><<<grid, kScatterChunk, smem, s>>>(p, g, prm, st, list, count, map, use_tma, use_ahead);
    else k_g2p2g<false><<<grid, kScatterChunk, smem, s>>>(p, g, prm, st, list, count, map, use_tma, use_ahead);
    MPMW_TRY_LAUNCH("k_g2p2g");
    k_stress_p2g_list<<<148 * 4, kBlock, 0, s>>>(p, g, prm, st, list, count);
    return check_launch("k_stress_p2g_list");
}

int launch_stress_p2g(const mpmw_particles_t &p, const mpmw_grid_t &g, const mpmw_params_t &prm, uint32_t *st,
                      void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (p.n == 0) return MPMW_OK;
    if (!ws || ws_bytes < g2p_workspace_bytes(p.n)) {
        set_error("stress_p2g: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  g2p_workspace_bytes(p.n));
        return MPMW_E_WORKSPACE;
    }
    const size_t smem = sizeof(ScatterShared);
    if (const int rc_ = reserve_fused_smem()) return rc_;
    int *count = static_cast<int *>(ws);
    int *list = reinterpret_cast<int *>(static_cast<char *>(ws) + 256);
    if (cudaMemsetAsync(count, 0, sizeof(int), s) != cudaSuccess) { set_error("stress_p2g: memset failed"); return MPMW_E_DEVICE; }
    k_stress_p2g<<<grid_for(p.n, kScatterChunk), kScatterChunk, smem, s>>>(p, g, prm, st, list, count);
    MPMW_TRY_LAUNCH("k_stress_p2g");
    k_stress_p2g_list<<<148 * 4, kBlock, 0, s>>>(p, g, prm, st, list, count);
    return check_launch("k_stress_p2g_list");
}

// ---------------------------------------------------------------------------
// batched scenes: one launch per kernel over many independent scenes
// ---------------------------------------------------------------------------
// The scenes' particles are concatenated in one set of SoA arrays (scene s owns
// the CTA-aligned particle range [offsets[s], offsets[s+1])); each scene keeps
// its own grid, parameters and grid tensor map.  mpmw_batch_prepare writes a
// table into the workspace: per scene its grid and parameters (128 B), and per
// CTA its scene, for the particle kernels and for the grid-node kernels.  A
// particle CTA reads its scene index once and one warp stages the scene's
// record in shared memory.  The tensor maps travel as a __grid_constant__
// kernel parameter (the usual home of a TMA descriptor: no proxy fence).
struct BatchScene {
    mpmw_grid_t grid;
    mpmw_params_t prm;
};
static_assert(sizeof(BatchScene) % 4 == 0 && sizeof(BatchScene) <= 32 * 4 * 2, "a scene record is staged by one warp");

struct BatchMaps {
    CUtensorMap tmap[MPMW_BATCH_MAX_SCENES];
};
static_assert(sizeof(BatchMaps) + sizeof(mpmw_particles_t) + 128 <= 32764, "the maps fit the kernel parameter space");

struct BatchRef {  // kernel argument: pointers into the prepared workspace
    const BatchScene *scene;
    const int *pcta_scene;  // particle CTA -> scene
    const int *ncta_scene;  // grid-node CTA -> scene
    const int *ncta_first;  // scene -> its first grid-node CTA
    int pcta_base;          // this launch covers particle CTAs pcta_base + blockIdx.x (a range of scenes)
    int ncta_base;          // ... and grid-node CTAs ncta_base + blockIdx.x
    int nscenes;            // scene indices read from the table are checked against it
    int use_tma;
};

// A scene index read from the table that is not one of the prepared scenes
// (a corrupted table): the CTA skips its work and reports it as MPMW_ST_OOB,
// so its particles do not silently stay where they are.
__device__ __forceinline__ bool bad_scene(int s, const BatchRef &R, uint32_t *status)
{
    if (s >= 0 && s < R.nscenes) return false;
    if (threadIdx.x == 0) raise_status(status, MPMW_ST_OOB);
    return true;
}

// Every thread of the CTA calls it: scene index of this particle CTA, and the
// scene's record copied into `rec` (published by the barrier); -1 (for the
// whole CTA, before any barrier, reported in *status) if the table holds no
// valid scene index.
__device__ __forceinline__ int stage_scene_at(const BatchRef &R, int pcta, BatchScene &rec, uint32_t *status)
{
    const int s = R.pcta_scene[pcta];
    if (bad_scene(s, R, status)) return -1;  // uniform: every thread read the same entry
    constexpr int kWords = (int)(sizeof(BatchScene) / 4);
    if (threadIdx.x < kWords)
        reinterpret_cast<uint32_t *>(&rec)[threadIdx.x] = reinterpret_cast<const uint32_t *>(&R.scene[s])[threadIdx.x];
    __syncthreads();
    return s;
}

__device__ __forceinline__ int stage_scene(const BatchRef &R, BatchScene &rec, uint32_t *status)
{
    return stage_scene_at(R, R.pcta_base + blockIdx.x, rec, status);
}

// Grid-node CTAs of the batch cover kBatchNodesPerCta nodes of one scene each
// (kBatchNodesPerThread per thread, kBlock apart), so the scene lookup is paid
// once per 2048 nodes.
constexpr int kBatchNodesPerThread = 8;
constexpr int kBatchNodesPerCta = kBlock * kBatchNodesPerThread;

// One grid-node entry b of the table (kBatchNodesPerCta nodes of one scene),
// by the blockDim.x threads of a CTA (kBatchNodesPerCta / blockDim.x nodes
// each, blockDim.x apart).
__device__ __forceinline__ void zero_grid_entry(const BatchRef &R, int b, uint32_t *status)
{
    const int s = R.ncta_scene[b];
    if (bad_scene(s, R, status)) return;
    const mpmw_grid_t G = R.scene[s].grid;
    const int64_t total = (int64_t)G.dims[0] * G.dims[1] * G.dims[2];
    const int64_t g0 = (int64_t)(b - R.ncta_first[s]) * kBatchNodesPerCta + threadIdx.x;
    const int per = kBatchNodesPerCta / (int)blockDim.x;
    for (int u = 0; u < per; ++u) {
        const int64_t g = g0 + (int64_t)u * blockDim.x;
        if (g < total) reinterpret_cast<float4 *>(G.mv)[g] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

template <int kGroup = kBatchNodesPerThread>
__device__ __forceinline__ void grid_update_entry(const BatchRef &R, int b, int zero_mv, uint32_t *status)
{
    const int s = R.ncta_scene[b];
    if (bad_scene(s, R, status)) return;
    const BatchScene B = R.scene[s];
    const int64_t g0 = (int64_t)(b - R.ncta_first[s]) * kBatchNodesPerCta + threadIdx.x;
    const int64_t total = (int64_t)B.grid.dims[0] * B.grid.dims[1] * B.grid.dims[2];
    const int per = kBatchNodesPerCta / (int)blockDim.x;
    for (int u0 = 0; u0 < per; u0 += kGroup) {
        // a group of nodes' accumulators is loaded before any store: the stores
        // go through pointers the compiler cannot tell apart from the loads, so
        // interleaving them would pay one memory latency per node
        float4 a[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            const int64_t g = g0 + (int64_t)(u0 + u) * blockDim.x;
            a[u] = g < total ? reinterpret_cast<const float4 *>(B.grid.mv)[g] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
            const int64_t g = g0 + (int64_t)(u0 + u) * blockDim.x;
            if (g < total) grid_update_apply(B.grid, B.prm, zero_mv, g, a[u]);
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_zero_grid_batch(const BatchRef R, uint32_t *status)
{
    zero_grid_entry(R, R.ncta_base + blockIdx.x, status);
}

// reset (may be NULL): the range's worklist count, set to 0 once
__global__ void __launch_bounds__(kBlock) k_grid_update_batch(const BatchRef R, int zero_mv, uint32_t *status,
                                                             int *reset)
{
    pdl_wait();
    pdl_trigger();
    if (reset && blockIdx.x == 0 && threadIdx.x == 0) *reset = 0;
    grid_update_entry(R, R.ncta_base + blockIdx.x, zero_mv, status);
}

__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_stress_p2g_batch(
    mpmw_particles_t P, const BatchRef R, uint32_t *status, int *svd_list, int *svd_count)
{
    __shared__ BatchScene B;
    if (stage_scene(R, B, status) < 0) return;
    stress_p2g_body(P, B.grid, B.prm, status, svd_list, svd_count,
                    (int64_t)(R.pcta_base + blockIdx.x) * kScatterChunk);
}

template <bool StoreStress>
__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_g2p2g_batch(
    mpmw_particles_t P, const BatchRef R, const __grid_constant__ BatchMaps M, uint32_t *status, int *svd_list,
    int *svd_count, int use_ahead)
{
    pdl_wait();
    pdl_trigger();
    __shared__ BatchScene B;
    const int s = stage_scene(R, B, status);
    if (s < 0) return;
    g2p2g_body<StoreStress>(P, B.grid, B.prm, status, svd_list, svd_count, &M.tmap[s], R.use_tma, use_ahead,
                            (int64_t)(R.pcta_base + blockIdx.x) * kScatterChunk);
}

// the batch's particle CTAs are the scatter's (kScatterChunk particles), so the
// scene table's CTA entries serve every batched particle kernel
__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_g2p_batch(mpmw_particles_t P, const BatchRef R,
                                                     const __grid_constant__ BatchMaps M, uint32_t *status,
                                                     int use_ahead)
{
    __shared__ BatchScene B;
    const int s = stage_scene(R, B, status);
    if (s < 0) return;
    g2p_body<false, kScatterChunk>(P, B.grid, B.prm, status, nullptr, nullptr, &M.tmap[s], R.use_tma, use_ahead,
                                   (int64_t)(R.pcta_base + blockIdx.x) * kScatterChunk);
}

// the listed (SVD-path) particles, by all threads of the grid
__device__ __forceinline__ void stress_p2g_list_batch_all(const mpmw_particles_t &P, const BatchRef &R,
                                                          uint32_t *status, const int *list, const int *count)
{
    const int cnt = *count;
    uint32_t bad = 0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        const int64_t p = list[q];
        if (p < 0 || p >= P.n) continue;
        const int s = R.pcta_scene[p / kScatterChunk];
        if (s < 0 || s >= R.nscenes) { bad |= MPMW_ST_OOB; continue; }
        const BatchScene &B = R.scene[s];
        stress_p2g_one(P, B.grid, B.prm, p, bad);
    }
    if (bad) raise_status(status, bad);
}

__global__ void __launch_bounds__(kBlock) k_stress_p2g_list_batch(mpmw_particles_t P, const BatchRef R,
                                                                 uint32_t *status, const int *__restrict__ list,
                                                                 const int *__restrict__ count)
{
    pdl_wait();
    pdl_trigger();
    stress_p2g_list_batch_all(P, R, status, list, count);
}


// ---------------------------------------------------------------------------
// The batch's fused substeps as one persistent kernel (cooperative launch):
// every fused substep (grid update, G2P -> return map -> P2G, the SVD
// worklist) of all scenes, phases separated by bounded grid barriers.  The
// prologue before it (grids cleared, the first return map and P2G) and the
// last grid update and G2P after it are the per-kernel launches.  Particle CTAs of the
// scene table are handed out as tiles from a ticket counter as CTAs free up
// (the scenes differ in size and in plastic work); grid-node entries are
// split evenly.  Each tile runs the body the per-kernel launches run.
// ---------------------------------------------------------------------------
struct BatchPersistArgs {
    mpmw_particles_t P;
    BatchRef R;
    uint32_t *status;
    int *list, *count;   // SVD worklist of the whole batch
    unsigned *arrive;    // grid-barrier arrivals
    unsigned *tickets;   // particle tiles drawn so far
    int nsteps;          // the run's substeps: its nsteps - 1 fused ones run here
    int pctas, nctas;    // particle tiles, grid-node entries
    int use_ahead;
};

// after every particle tile: the tile's shared-memory writes (generic proxy)
// are ordered before the next tile's bulk and TMA copies into the same bytes
// (async proxy), and no thread is still in the tile.  Returns false (for the
// whole CTA) once the launch has reported a copy timeout that was not set
// when it started: a copy may still be in flight, so the CTA stops.
__device__ __forceinline__ bool batch_tile_done(uint32_t *status, uint32_t st0, int *s_stop)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t now = status ? *reinterpret_cast<volatile uint32_t *>(status) : 0u;
        *s_stop = (now & MPMW_ST_TIMEOUT) && !(st0 & MPMW_ST_TIMEOUT);
    }
    __syncthreads();
    return *s_stop == 0;
}

__global__ void __launch_bounds__(kScatterChunk, kScatterCtasPerSm) k_batch_persistent(
    const __grid_constant__ BatchPersistArgs A, const __grid_constant__ BatchMaps M)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ BatchScene B;
    __shared__ int s_ok, s_tile, s_stop;
    // the fused body's shared layout (as g2p2g_body places it), for its barriers
    G2P2GShared &S = *reinterpret_cast<G2P2GShared *>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    const uint32_t st0 = A.status ? *reinterpret_cast<volatile uint32_t *>(A.status) : 0u;
    const int64_t n = A.P.n;
    unsigned tick = 0;  // tickets drawn by the earlier tiled phases
    const unsigned per_phase = (unsigned)A.pctas + gridDim.x;
    for (int step = 0; step + 1 < A.nsteps; ++step) {
        for (int b = blockIdx.x; b < A.nctas; b += gridDim.x) grid_update_entry<4>(A.R, b, 1, A.status);
        if (blockIdx.x == 0 && threadIdx.x == 0) *A.count = 0;  // the list phase that read it is over
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        const bool store = step + 2 == A.nsteps;  // the last fused substep writes the stress
        for (int t = draw_tile(A.tickets, tick, &s_tile); t < A.pctas; t = draw_tile(A.tickets, tick, &s_tile)) {
            const int sc = stage_scene_at(A.R, t, B, A.status);
            const int64_t p0 = (int64_t)t * kScatterChunk;
            // one body, the stress store chosen at run time (a uniform branch)
            if (sc >= 0)
                g2p2g_body<false>(A.P, B.grid, B.prm, A.status, A.list, A.count, &M.tmap[sc], A.R.use_tma,
                                  A.use_ahead, p0, store);
            __syncthreads();
            if (sc >= 0 && threadIdx.x == 0) {
                // the body initialised these barriers; their bytes are reused
                mbar_inval(&S.g.bar);
                if (A.use_ahead && p0 + kScatterChunk <= n) mbar_inval(&S.pbar);
            }
            if (!batch_tile_done(A.status, st0, &s_stop)) return;
        }
        tick += per_phase;
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        stress_p2g_list_batch_all(A.P, A.R, A.status, A.list, A.count);
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
    }
}

namespace {
// Workspace layout of a batch: the SVD worklist (n ints; a range of scenes
// lists its particles in its own part, from the range's first particle on),
// one worklist count per scene (a range uses its first scene's), the scene
// records, the three CTA tables, then the persistent form's barrier and
// ticket counters.
struct BatchLayout {
    size_t list, counts, scenes, pcta, ncta, nfirst, sync, total;
};
size_t round256(size_t b) { return (b + 255) / 256 * 256; }
BatchLayout batch_layout(int64_t n, int nscenes, int64_t nctas)
{
    BatchLayout L;
    L.list = 0;
    L.counts = round256((size_t)n * sizeof(int));
    L.scenes = L.counts + round256((size_t)nscenes * sizeof(int));
    L.pcta = L.scenes + round256((size_t)nscenes * sizeof(BatchScene));
    L.ncta = L.pcta + round256((size_t)(n / kScatterChunk) * sizeof(int));
    L.nfirst = L.ncta + round256((size_t)nctas * sizeof(int));
    L.sync = L.nfirst + round256((size_t)(nscenes + 1) * sizeof(int));  // the persistent form's counters
    L.total = L.sync + 256;
    return L;
}
int64_t scene_node_ctas(const mpmw_grid_t &g)
{
    return grid_for((int64_t)g.dims[0] * g.dims[1] * g.dims[2], kBatchNodesPerCta);
}
int64_t batch_node_ctas(const mpmw_grid_t *grids, int nscenes)
{
    int64_t c = 0;
    for (int k = 0; k < nscenes; ++k) c += scene_node_ctas(grids[k]);
    return c;
}
// what a prepared workspace holds, for mpmw_batch_run_substeps
struct BatchPrepared {
    int64_t n;
    int nscenes, pctas, nctas, use_tma, use_ahead, use_ahead_g2p;
    int tma_avail = -1, ahead_avail = 0, ahead_g2p_avail = 0;  // what prepare found usable (set_batch_options)
    BatchLayout L;
    std::shared_ptr<BatchMaps> maps;
    std::vector<int> pfirst, nfirst;  // first particle / grid-node CTA of each scene (+ the totals)
};
std::mutex g_batch_mu;
std::unordered_map<const void *, BatchPrepared> g_batches;
}  // namespace

size_t batch_workspace_bytes(const mpmw_grid_t *grids, int nscenes, int64_t n)
{
    return batch_layout(n, nscenes, batch_node_ctas(grids, nscenes)).total;
}

// Writes the scene table into the workspace (synchronizes the stream) and
// remembers the batch's launch sizes.  The caller has checked the arguments.
int prepare_batch(const mpmw_particles_t &p, const mpmw_grid_t *grids, const mpmw_params_t *prms,
                  const int64_t *offsets, int nscenes, void *ws, size_t ws_bytes, cudaStream_t s)
{
    const int64_t nctas = batch_node_ctas(grids, nscenes);
    const BatchLayout L = batch_layout(p.n, nscenes, nctas);
    if (nscenes > MPMW_BATCH_MAX_SCENES) {
        set_error("batch: %d scenes (at most %d per batch)", nscenes, MPMW_BATCH_MAX_SCENES);
        return MPMW_E_ARG;
    }
    if (reinterpret_cast<uintptr_t>(ws) & 15u) { set_error("batch: the workspace must be 16-byte aligned"); return MPMW_E_ARG; }
    if (ws_bytes < L.total) {
        set_error("batch: workspace of %zu bytes is smaller than the %zu required", ws_bytes, L.total);
        return MPMW_E_WORKSPACE;
    }
    const size_t tbytes = L.total - L.scenes;
    std::vector<unsigned char> host(tbytes, 0);
    BatchScene *sc = reinterpret_cast<BatchScene *>(host.data());
    int *pcta = reinterpret_cast<int *>(host.data() + (L.pcta - L.scenes));
    int *ncta = reinterpret_cast<int *>(host.data() + (L.ncta - L.scenes));
    int *nfirst = reinterpret_cast<int *>(host.data() + (L.nfirst - L.scenes));
    auto maps = std::make_shared<BatchMaps>();
    memset(maps.get(), 0, sizeof(BatchMaps));
    int use_tma = 1, c = 0;
    for (int k = 0; k < nscenes; ++k) {
        if (!cached_grid_map(grids[k], &maps->tmap[k])) use_tma = 0;
        sc[k].grid = grids[k];
        sc[k].prm = prms[k];
        static_assert(256 % kScatterChunk == 0, "scene offsets (multiples of 256) fall on particle-CTA boundaries");
        for (int64_t b = offsets[k] / kScatterChunk; b < offsets[k + 1] / kScatterChunk; ++b) pcta[b] = k;
        nfirst[k] = c;
        const int nc = (int)scene_node_ctas(grids[k]);
        for (int b = 0; b < nc; ++b) ncta[c + b] = k;
        c += nc;
    }
    nfirst[nscenes] = c;
    unsigned char *dst = static_cast<unsigned char *>(ws) + L.scenes;
    if (cudaMemcpyAsync(dst, host.data(), tbytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        set_error("batch: copying the scene table failed");
        return MPMW_E_DEVICE;
    }
    BatchPrepared bp;
    bp.n = p.n;
    bp.nscenes = nscenes;
    bp.pctas = (int)(p.n / kScatterChunk);
    bp.nctas = (int)nctas;
    bp.use_tma = use_tma;
    bp.use_ahead = g2p2g_ahead_ok(p) ? 1 : 0;
    bp.use_ahead_g2p = p.F && p.n % 4 == 0 && (reinterpret_cast<uintptr_t>(p.F) & 15u) == 0 ? 1 : 0;
    bp.L = L;
    bp.maps = maps;
    bp.pfirst.resize(nscenes + 1);
    bp.nfirst.assign(nfirst, nfirst + nscenes + 1);
    for (int k = 0; k <= nscenes; ++k) bp.pfirst[k] = (int)(offsets[k] / kScatterChunk);
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if (g_batches.size() > 256) g_batches.clear();
    g_batches[ws] = bp;
    return MPMW_OK;
}

// The launch options of a prepared batch (what ConcatBatch.tune searches):
// the G2P grid tile by TMA (else the gather reads the grid through L1) and the
// bulk read-ahead of the particle fields (else plain loads).  Either can only
// be turned off where prepare_batch found it usable.  Returns false if the
// workspace was not prepared.
bool set_batch_options(const void *ws, int gather_tile, int read_ahead)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    auto it = g_batches.find(ws);
    if (it == g_batches.end()) return false;
    BatchPrepared &bp = it->second;
    if (bp.tma_avail < 0) { bp.tma_avail = bp.use_tma; bp.ahead_avail = bp.use_ahead; bp.ahead_g2p_avail = bp.use_ahead_g2p; }
    bp.use_tma = gather_tile ? bp.tma_avail : 0;
    bp.use_ahead = read_ahead ? bp.ahead_avail : 0;
    bp.use_ahead_g2p = read_ahead ? bp.ahead_g2p_avail : 0;
    return true;
}

// per device: the batched kernels' shared-memory attribute is set (several host
// threads may launch batches at once; setting it twice is harmless)
static std::atomic<bool> g_batch_attr[64];
std::atomic<int64_t> g_batch_persistent_launches{0};
int64_t batch_persistent_launches() { return g_batch_persistent_launches.load(); }

// The fused schedule of mpmw_run_substeps over the scenes [first, last) of a
// batch that prepare_batch wrote into this workspace (last < 0: to the end).
// Disjoint scene ranges touch disjoint particles, grids and worklists, so they
// may run concurrently on different streams.
int launch_batch_substeps(const mpmw_particles_t &p, int first, int last, int nsteps, uint32_t *st, void *ws,
                          size_t ws_bytes, cudaStream_t s)
{
    BatchPrepared bp;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        auto it = g_batches.find(ws);
        if (it == g_batches.end()) { set_error("batch: the workspace was not prepared (mpmw_batch_prepare)"); return MPMW_E_ARG; }
        bp = it->second;
    }
    if (bp.n != p.n || ws_bytes < bp.L.total) {
        set_error("batch: the workspace was prepared for %lld particles in %zu bytes", (long long)bp.n, bp.L.total);
        return MPMW_E_ARG;
    }
    if (last < 0) last = bp.nscenes;
    if (first < 0 || first >= last || last > bp.nscenes) {
        set_error("batch: scene range [%d, %d) outside the %d prepared scenes", first, last, bp.nscenes);
        return MPMW_E_ARG;
    }
    if (nsteps == 0 || p.n == 0) return MPMW_OK;
    const size_t smem = sizeof(G2P2GShared) + 128;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_error("batch: no current device"); return MPMW_E_DEVICE; }
    if (dev >= 0 && dev < 64 && !g_batch_attr[dev].load(std::memory_order_acquire)) {
        if (cudaFuncSetAttribute(k_g2p2g_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_g2p2g_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(k_stress_p2g_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(ScatterShared)) != cudaSuccess) {
            set_error("batch: cannot reserve %zu bytes of shared memory", smem);
            return MPMW_E_DEVICE;
        }
        g_batch_attr[dev].store(true, std::memory_order_release);
    }
    unsigned char *base = static_cast<unsigned char *>(ws);
    BatchRef R;
    R.scene = reinterpret_cast<const BatchScene *>(base + bp.L.scenes);
    R.pcta_scene = reinterpret_cast<const int *>(base + bp.L.pcta);
    R.ncta_scene = reinterpret_cast<const int *>(base + bp.L.ncta);
    R.ncta_first = reinterpret_cast<const int *>(base + bp.L.nfirst);
    R.pcta_base = bp.pfirst[first];
    R.ncta_base = bp.nfirst[first];
    R.nscenes = bp.nscenes;
    R.use_tma = bp.use_tma;
    int *count = reinterpret_cast<int *>(base + bp.L.counts) + first;
    int *list = reinterpret_cast<int *>(base + bp.L.list) + (int64_t)bp.pfirst[first] * kScatterChunk;
    const unsigned pctas = (unsigned)(bp.pfirst[last] - bp.pfirst[first]);
    const unsigned nctas = (unsigned)(bp.nfirst[last] - bp.nfirst[first]);
    auto reset_count = [&]() -> int {
        if (cudaMemsetAsync(count, 0, sizeof(int), s) != cudaSuccess) { set_error("batch: memset failed"); return MPMW_E_DEVICE; }
        return MPMW_OK;
    };
    // prologue: every grid cleared, substep 1's return map and P2G
    k_zero_grid_batch<<<nctas, kBlock, 0, s>>>(R, st);
    MPMW_TRY_LAUNCH("k_zero_grid_batch");
    if (reset_count() != MPMW_OK) return MPMW_E_DEVICE;
    k_stress_p2g_batch<<<pctas, kScatterChunk, sizeof(ScatterShared), s>>>(p, R, st, list, count);
    MPMW_TRY_LAUNCH("k_stress_p2g_batch");
    k_stress_p2g_list_batch<<<148 * 4, kBlock, 0, s>>>(p, R, st, list, count);
    MPMW_TRY_LAUNCH("k_stress_p2g_list_batch");
    for (int step = 0; step < nsteps; ++step) {
        if (step < nsteps - 1) {
            // grid pass (which also resets the worklist count) -> fused kernel
            // -> worklist, as programmatic dependent launches (each waits for
            // its predecessor before it reads anything)
            cudaError_t e = launch_pdl(k_grid_update_batch, nctas, kBlock, 0, s, R, 1, st, count);
            if (e == cudaSuccess)
                e = step + 1 == nsteps - 1
                        ? launch_pdl(k_g2p2g_batch<true>, pctas, kScatterChunk, smem, s, p, R, *bp.maps, st, list,
                                     count, bp.use_ahead)
                        : launch_pdl(k_g2p2g_batch<false>, pctas, kScatterChunk, smem, s, p, R, *bp.maps, st, list,
                                     count, bp.use_ahead);
            if (e == cudaSuccess)
                e = launch_pdl(k_stress_p2g_list_batch, 148 * 4, kBlock, 0, s, p, R, st, (const int *)list,
                               (const int *)count);
            if (e != cudaSuccess) {
                set_error("batch: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
                return MPMW_E_DEVICE;
            }
        } else {
            k_grid_update_batch<<<nctas, kBlock, 0, s>>>(R, 0, st, nullptr);
            MPMW_TRY_LAUNCH("k_grid_update_batch");
            k_g2p_batch<<<pctas, kScatterChunk, 0, s>>>(p, R, *bp.maps, st, bp.use_ahead_g2p);
            MPMW_TRY_LAUNCH("k_g2p_batch");
        }
    }
    return MPMW_OK;
}

// CTAs of the persistent batch kernel's cooperative grid on the current
// device (0: it cannot be launched there)
static int batch_persist_capacity(size_t smem)
{
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 0;
    if (dev < 64) {
        const int c = cache[dev].load();
        if (c != 0) return c > 0 ? c : 0;
    }
    int coop = 0, sms = 0, per_sm = 0, cap = -1;
    if (cudaFuncSetAttribute(k_batch_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persistent, kScatterChunk, smem) ==
            cudaSuccess &&
        per_sm > 0)
        cap = per_sm * sms;
    cudaGetLastError();
    if (dev < 64) cache[dev].store(cap);
    return cap > 0 ? cap : 0;
}

// All scenes of a prepared batch, nsteps substeps: the prologue, the fused
// substeps in one persistent launch, then the last grid update and G2P.
int launch_batch_persistent(const mpmw_particles_t &p, int nsteps, uint32_t *st, void *ws, size_t ws_bytes,
                            cudaStream_t s)
{
    BatchPrepared bp;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        auto it = g_batches.find(ws);
        if (it == g_batches.end()) { set_error("batch: the workspace was not prepared (mpmw_batch_prepare)"); return MPMW_E_ARG; }
        bp = it->second;
    }
    if (bp.n != p.n || ws_bytes < bp.L.total) {
        set_error("batch: the workspace was prepared for %lld particles in %zu bytes", (long long)bp.n, bp.L.total);
        return MPMW_E_ARG;
    }
    if (nsteps == 0 || p.n == 0) return MPMW_OK;
    const size_t smem = sizeof(G2P2GShared) + 128;
    static_assert(sizeof(G2P2GShared) + 128 >= sizeof(ScatterShared), "the stress + P2G phase fits the same buffer");
    const int cap = batch_persist_capacity(smem);
    if (cap <= 0) { set_error("batch: the device cannot run the persistent batch kernel"); return MPMW_E_DEVICE; }
    unsigned char *base = static_cast<unsigned char *>(ws);
    BatchPersistArgs A;
    memset(&A, 0, sizeof(A));
    A.P = p;
    A.R.scene = reinterpret_cast<const BatchScene *>(base + bp.L.scenes);
    A.R.pcta_scene = reinterpret_cast<const int *>(base + bp.L.pcta);
    A.R.ncta_scene = reinterpret_cast<const int *>(base + bp.L.ncta);
    A.R.ncta_first = reinterpret_cast<const int *>(base + bp.L.nfirst);
    A.R.pcta_base = 0;
    A.R.ncta_base = 0;
    A.R.nscenes = bp.nscenes;
    A.R.use_tma = bp.use_tma;
    A.status = st;
    A.list = reinterpret_cast<int *>(base + bp.L.list);
    A.count = reinterpret_cast<int *>(base + bp.L.counts);
    A.arrive = reinterpret_cast<unsigned *>(base + bp.L.sync);
    A.tickets = A.arrive + 1;
    A.nsteps = nsteps;
    A.pctas = bp.pctas;
    A.nctas = bp.nctas;
    A.use_ahead = bp.use_ahead;
    if (cudaMemsetAsync(base + bp.L.sync, 0, 2 * sizeof(unsigned), s) != cudaSuccess ||
        cudaMemsetAsync(A.count, 0, sizeof(int), s) != cudaSuccess) {
        set_error("batch: memset failed");
        return MPMW_E_DEVICE;
    }
    BatchRef R = A.R;
    k_zero_grid_batch<<<(unsigned)bp.nctas, kBlock, 0, s>>>(R, st);
    MPMW_TRY_LAUNCH("k_zero_grid_batch");
    k_stress_p2g_batch<<<(unsigned)bp.pctas, kScatterChunk, sizeof(ScatterShared), s>>>(p, R, st, A.list, A.count);
    MPMW_TRY_LAUNCH("k_stress_p2g_batch");
    k_stress_p2g_list_batch<<<148 * 4, kBlock, 0, s>>>(p, R, st, A.list, A.count);
    MPMW_TRY_LAUNCH("k_stress_p2g_list_batch");
    const int grid = bp.pctas < cap ? (bp.pctas > 0 ? bp.pctas : 1) : cap;
    void *args[] = {&A, bp.maps.get()};
    if (cudaLaunchCooperativeKernel((const void *)k_batch_persistent, dim3((unsigned)grid), dim3(kScatterChunk), args,
                                    smem, s) != cudaSuccess) {
        set_error("batch: cooperative launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        return MPMW_E_DEVICE;
    }
    g_batch_persistent_launches.fetch_add(1);
    k_grid_update_batch<<<(unsigned)bp.nctas, kBlock, 0, s>>>(R, 0, st, nullptr);
    MPMW_TRY_LAUNCH("k_grid_update_batch");
    k_g2p_batch<<<(unsigned)bp.pctas, kScatterChunk, 0, s>>>(p, R, *bp.maps, st, bp.use_ahead_g2p);
    MPMW_TRY_LAUNCH("k_g2p_batch");
    return MPMW_OK;
}

}  // namespace mpmw
