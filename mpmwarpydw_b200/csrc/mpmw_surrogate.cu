// mpmw_surrogate.cu -- the stress phase with the learned return map
// (no counterpart in the reference; the plain map is utils/mpmRoutines.py:314-453,
// the stress phase :229-312).
//
// Three kernels per call:
//   k_surr_classify  per active MPM particle, exactly as the plain stress phase
//                    for: deformations outside the tensor form's range (SVD
//                    path), elastic trials, and trials that set D = 1 (ys < 0
//                    or negative yield).  Plastic trials in range are listed
//                    with their principal log strains e, eigenvectors Q and
//                    surrogate features.
//   k_mlp_infer_tc   the network on the listed features (tensor cores).
//   k_surr_finish    the return from the network's ratios (include/mpmw_mlp.h):
//                    rho = exp(y[0]), dgamma = n exp(y[1]) + 1e-6 with
//                    n = |dev e|, e_ret = e + (rho n/(n + 1e-6) - 1) dev e +
//                    y[2] dgamma, d_acc = y[3] dgamma;
//                    a gate on the return's defining identities (the yield
//                    condition's deviatoric norm and the flow rule's volumetric
//                    part and strain increment): the surrogate's principal
//                    stresses and increment against the state they define,
//                    each within `gate_tol`, else the exact closed-form return;
//                    an audit of a hashed fraction of the surrogate's returns
//                    (before the gate) against the exact return (relative
//                    error of the principal stresses: largest, sum, count
//                    within 1e-3);
//                    then damage, phase transition, hardening, F and the
//                    Kirchhoff + Kelvin-Voigt stress as the plain path.
#include "mpmw_common.cuh"
#include "mpmw_internal.cuh"
#include "mpmw_math.cuh"
#include "mpmw_stress.cuh"
#include "../../include/mpmw_mlp.h"

namespace mpmw {

int launch_mlp_infer_tc_dev(const void *packed, const float *params, const float *x, int64_t n_max, const int *n_dev,
                            float *y, uint32_t *status, cudaStream_t s);

namespace {

struct SurrWork {
    int *count;
    int *idx;       // [n] particle
    float *feat;    // [n][8]
    float *out;     // [n][4]
    float *eq;      // [n][12]: e (3), Q (9)
};

__host__ __device__ inline size_t al256(size_t b) { return (b + 255) / 256 * 256; }

SurrWork carve(void *ws, int64_t n)
{
    char *w = static_cast<char *>(ws);
    SurrWork s;
    s.count = reinterpret_cast<int *>(w); w += 256;
    s.idx = reinterpret_cast<int *>(w); w += al256(4 * (size_t)n);
    s.feat = reinterpret_cast<float *>(w); w += al256(32 * (size_t)n);
    s.out = reinterpret_cast<float *>(w); w += al256(16 * (size_t)n);
    s.eq = reinterpret_cast<float *>(w);
    return s;
}

// strain invariants of the trial state (tensor form), as small_strain_update
struct Trial {
    float eps[6], dev[6], tr, dev_norm, pst, yield_eff, mu, lam, ys, alpha, D;
};

__device__ __forceinline__ bool trial_in_range(const float *Ft, float *eps)
{
    float G[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = Ft[k] - ((k & 3) == 0 ? 1.f : 0.f);
    float X[6];
    const int rr[6] = {0, 1, 2, 0, 0, 1}, cc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const int r = rr[e], c = cc[e];
        X[e] = fma_(G[3 * r + 0], G[3 * c + 0], fma_(G[3 * r + 1], G[3 * c + 1],
                    fma_(G[3 * r + 2], G[3 * c + 2], G[3 * r + c] + G[3 * c + r])));
    }
    if (!(sym_ddot(X, X) <= 4e-4f)) return false;
    const float det = Ft[0] * (Ft[4] * Ft[8] - Ft[5] * Ft[7]) - Ft[1] * (Ft[3] * Ft[8] - Ft[5] * Ft[6]) +
                      Ft[2] * (Ft[3] * Ft[7] - Ft[4] * Ft[6]);
    if (!(det > 0.f)) return false;
    float Pm[6], Q[6], L[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) Pm[e] = -0.25f * X[e] + (e < 3 ? (1.f / 3.f) : 0.f);
    sym_mul(X, Pm, Q);
    Q[0] -= 0.5f; Q[1] -= 0.5f; Q[2] -= 0.5f;
    sym_mul(X, Q, Pm);
    Pm[0] += 1.f; Pm[1] += 1.f; Pm[2] += 1.f;
    sym_mul(X, Pm, L);
#pragma unroll
    for (int e = 0; e < 6; ++e) eps[e] = 0.5f * L[e];
    return true;
}

__device__ __forceinline__ void make_trial(const mpmw_particles_t &P, int64_t p, const float *eps, Trial &T)
{
#pragma unroll
    for (int e = 0; e < 6; ++e) T.eps[e] = eps[e];
    T.mu = P.mu[p]; T.lam = P.lam[p]; T.ys = P.ys[p]; T.alpha = P.alpha[p]; T.D = P.damage[p];
    T.tr = (eps[0] + eps[1]) + eps[2];
    const float mean = T.tr / 3.f;
    T.dev[0] = eps[0] - mean; T.dev[1] = eps[1] - mean; T.dev[2] = eps[2] - mean;
    T.dev[3] = eps[3]; T.dev[4] = eps[4]; T.dev[5] = eps[5];
    T.dev_norm = sqrtf(sym_ddot(T.dev, T.dev));
    const float twomu = 2.f * T.mu;
    T.pst = fma_(twomu / 3.f, T.tr, T.lam * T.tr);
    T.yield_eff = (1.f - T.D) * (T.ys - T.alpha * T.pst);
}

__device__ __forceinline__ uint32_t audit_hash(uint64_t x)
{
    x ^= x >> 33; x *= 0xFF51AFD7ED558CCDull; x ^= x >> 33; x *= 0xC4CEB9FE1A85EC53ull; x ^= x >> 33;
    return (uint32_t)x;
}

}  // namespace

__global__ void __launch_bounds__(kBlock) k_surr_classify(mpmw_particles_t P, float eff, SurrWork W)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = P.n;
    if (p >= n || P.active[p] != 1 || !(P.material[p] <= 1)) return;
    float Ft[9], Cg[9], eps[6];
    load9(P.F_trial, n, p, Ft);
    load9(P.C, n, p, Cg);
    bool listed = false;
    if (trial_in_range(Ft, eps)) {
        Trial T;
        make_trial(P, p, eps, T);
        const bool d_one = T.ys < 0.f || T.yield_eff < 0.f;
        const bool plastic = (2.f * T.mu) * T.dev_norm > T.yield_eff;
        if (plastic && !d_one && T.dev_norm > 0.f && T.D <= MPMW_SURR_D_MAX) {
            float A[9], lam[3], Q[9];
            sym_to_full(eps, A);
            sym_eigen3(A, lam, Q);
            const float mag = sqrtf(fma_(lam[0], lam[0], fma_(lam[1], lam[1], lam[2] * lam[2])));
            const float y = T.ys / (2.f * T.mu);
            const int slot = atomicAdd(W.count, 1);
            W.idx[slot] = (int)p;
            float *f = W.feat + 8 * (int64_t)slot;
            f[0] = lam[0] / mag; f[1] = lam[1] / mag; f[2] = lam[2] / mag;
            f[3] = log10f(mag / y);
            f[4] = T.alpha; f[5] = 0.3f * T.alpha; f[6] = log1pf(-T.D);
            f[7] = T.lam / (2.f * (T.lam + T.mu));
            float *q = W.eq + 12 * (int64_t)slot;
            q[0] = lam[0]; q[1] = lam[1]; q[2] = lam[2];
#pragma unroll
            for (int k = 0; k < 9; ++k) q[3 + k] = Q[k];
            listed = true;
        }
    }
    if (!listed) {
        // exactly the plain stress phase (tensor form when it applies, else SVD)
        float Fo[9], out[9];
        stress_particle<false>(P, eff, MPMW_STRESS_AUTO, p, Ft, Cg, nullptr, nullptr, Fo, out);
        store9(P.F, n, p, Fo);
        store_sym6(P.stress, n, p, out);
    }
}

// stats: [0] listed (surrogate candidates), [1] gate fallbacks, [2] audited,
// [3] largest audited relative stress error (float bits, atomicMax on the bits
// of a non-negative float), [4] sum of audited relative errors (float),
// [5] audited with relative error <= 1e-3, [6] audited and accepted by the
// gate, [7] largest audited relative stress error among those accepted
__global__ void __launch_bounds__(kBlock) k_surr_finish(mpmw_particles_t P, float eff, SurrWork W, float gate_tol,
                                                        int audit_per_mille, uint64_t audit_seed, uint32_t *stats)
{
    const int cnt = *W.count;
    const int64_t n = P.n;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += gridDim.x * blockDim.x) {
        const int64_t p = W.idx[q];
        float Ft[9], Cg[9], eps[6];
        load9(P.F_trial, n, p, Ft);
        load9(P.C, n, p, Cg);
        trial_in_range(Ft, eps);  // recomputes eps exactly as classified
        Trial T;
        make_trial(P, p, eps, T);
        const float *eq = W.eq + 12 * (int64_t)q;
        const float e[3] = {eq[0], eq[1], eq[2]};
        float Q[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) Q[k] = eq[3 + k];
        const float *y = W.out + 4 * (int64_t)q;
        const float em = (e[0] + e[1] + e[2]) / 3.f;
        const float ed[3] = {e[0] - em, e[1] - em, e[2] - em};
        const float nd = sqrtf(fma_(ed[0], ed[0], fma_(ed[1], ed[1], ed[2] * ed[2])));
        const float edn = nd + 1e-6f;
        // the network's return: deviator scaled by rho n / (n + 1e-6), plastic
        // multiplier n (1 - rho) + 1e-6 (both ratios predicted in log form)
        const float rho = expf(y[0]);
        const float dg = fma_(nd, expf(y[1]), 1e-6f);
        const float sdev = rho * (nd / edn) - 1.f;
        float er[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) er[k] = fma_(sdev, ed[k], e[k]) + y[2] * dg;
        float dacc = y[3] * dg;
        // exact return quantities of the trial (closed form)
        const float twomu = 2.f * T.mu;
        const float dg_ex = edn - T.yield_eff / twomu;
        const float beta = 0.3f * T.alpha;
        // the state the return's identities define: the yield condition fixes the
        // returned deviatoric norm (yield / 2 mu, scaled by n / (n + 1e-6) as the
        // reference's radial return does), the non-associated flow rule the
        // volumetric part (beta dgamma) and the accumulated-strain increment
        // (sqrt(2/3) dgamma)
        float ex[3];
        const float f_ex = dg_ex / edn, vc_ex = beta * dg_ex;
#pragma unroll
        for (int k = 0; k < 3; ++k) ex[k] = fma_(-f_ex, ed[k], e[k]) + vc_ex;
        // gate: the surrogate's principal stresses against that state (relative,
        // norm-wise) and its accumulated-strain increment (relative to the
        // larger of the increment and the yield strain), each within gate_tol
        float num = 0.f, den = 0.f;
        {
            const float ts = T.lam * (er[0] + er[1] + er[2]), tx = T.lam * (ex[0] + ex[1] + ex[2]);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float a = fma_(twomu, er[k], ts), b = fma_(twomu, ex[k], tx);
                num += (a - b) * (a - b);
                den += b * b;
            }
        }
        const float ysc = fmaxf(T.yield_eff / twomu, 1e-12f);
        const float r_stress = sqrtf(num) / fmaxf(sqrtf(den), 1e-30f);
        const float r_acc = fabsf(dacc - sqrtf(2.f / 3.f) * dg_ex) / (sqrtf(2.f / 3.f) * fmaxf(dg_ex, ysc));
        const bool ok = dg > 0.f && r_stress <= gate_tol && r_acc <= gate_tol && isfinite(er[0]) &&
                        isfinite(er[1]) && isfinite(er[2]) && isfinite(dacc);
        if (audit_per_mille > 0 && (int)(audit_hash(audit_seed ^ (uint64_t)p) % 1000u) < audit_per_mille) {
            // audit the surrogate's own return (before the gate) against the exact one:
            // relative error of the principal stresses
            const float ts = T.lam * (er[0] + er[1] + er[2]), tx = T.lam * (ex[0] + ex[1] + ex[2]);
            float num = 0.f, den = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float a = fma_(twomu, er[k], ts), b = fma_(twomu, ex[k], tx);
                num += (a - b) * (a - b);
                den += b * b;
            }
            float rel = sqrtf(num) / fmaxf(sqrtf(den), 1e-30f);
            if (!isfinite(rel)) rel = 3.0e38f;
            atomicAdd(&stats[2], 1u);
            atomicMax(&stats[3], __float_as_uint(rel));
            atomicAdd(reinterpret_cast<float *>(&stats[4]), rel);
            if (rel <= 1e-3f) atomicAdd(&stats[5], 1u);
            if (ok) {
                atomicAdd(&stats[6], 1u);
                atomicMax(&stats[7], __float_as_uint(rel));
            }
        }
        if (!ok) {
            atomicAdd(&stats[1], 1u);
            er[0] = ex[0]; er[1] = ex[1]; er[2] = ex[2];
            dacc = sqrtf(2.f / 3.f) * dg_ex;
        }
        atomicAdd(&stats[0], 1u);
        // damage, transition, hardening (utils/mpmRoutines.py:361-440)
        float D = T.D;
        P.acc_strain[p] = P.acc_strain[p] + dacc;
        const float sc = P.strain_criteria[p];
        if (sc > 0.f) D = rmin(1.f, D + dacc / sc);
        else D = 1.f;
        P.damage[p] = D;
        float out[9], Tk[9];
        float Fo[9];
        if (D >= 1.f && P.material[p] == 1) {
            P.material[p] = 2;
            float xx[3], vv[3];
            load3(P.x, n, p, xx);
            load3(P.v, n, p, vv);
            store3(P.x_pc, n, p, xx);
            float tau[6];
            const float ltr = T.lam * T.tr;
#pragma unroll
            for (int k = 0; k < 6; ++k) tau[k] = fma_(twomu, T.eps[k], k < 3 ? ltr : 0.f);
            const float u = 0.5f * sym_ddot(tau, T.eps);
            const float vexp = sqrtf(((2.f * eff) * u) / P.density[p]);
            float vb[3] = {vv[0] + 1e-12f, vv[1] + 1e-12f, vv[2] + 1e-12f};
            float vd[3];
            normalize3(vb, vd);
            vv[0] = vv[0] + vexp * vd[0]; vv[1] = vv[1] + vexp * vd[1]; vv[2] = vv[2] + vexp * vd[2];
            store3(P.v_pc, n, p, vv);
            store3(P.v, n, p, vv);
            P.ys[p] = 0.f; P.mu[p] = 0.f; P.lam[p] = 0.f; P.alpha[p] = 0.f;
#pragma unroll
            for (int k = 0; k < 9; ++k) { Tk[k] = 0.f; Fo[k] = Ft[k]; }
        } else {
            const float dsy = (twomu * (P.hardening[p] - P.softening[p])) * (ok ? dg : dg_ex);
            P.ys[p] = rmax(0.f, T.ys + dsy);
            // eps_ret = Q diag(e_ret) Q^T, F_e = Q diag(exp(e_ret - e)) Q^T F_trial,
            // tau = 2 mu eps_ret + lam tr(eps_ret) I
            const float trr = (er[0] + er[1]) + er[2];
            float M[9], Ex[9];
            const float tk[3] = {fma_(twomu, er[0], T.lam * trr), fma_(twomu, er[1], T.lam * trr),
                                 fma_(twomu, er[2], T.lam * trr)};
            const float xk[3] = {expf(er[0] - e[0]), expf(er[1] - e[1]), expf(er[2] - e[2])};
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float a = 0.f, b = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        a = fma_(Q[3 * r + k] * tk[k], Q[3 * c + k], a);
                        b = fma_(Q[3 * r + k] * xk[k], Q[3 * c + k], b);
                    }
                    M[3 * r + c] = a;
                    Ex[3 * r + c] = b;
                }
            matmul3(Ex, Ft, Fo);
#pragma unroll
            for (int k = 0; k < 9; ++k) Tk[k] = M[k];
        }
        add_viscous(Tk, Cg, P.eta_shear[p], P.eta_bulk[p], out);
        store9(P.F, n, p, Fo);
        store_sym6(P.stress, n, p, out);
    }
}

size_t surrogate_workspace_bytes(int64_t n)
{
    n = n < 0 ? 0 : n;
    return 256 + al256(4 * (size_t)n) + al256(32 * (size_t)n) + al256(16 * (size_t)n) + al256(48 * (size_t)n);
}

}  // namespace mpmw

using namespace mpmw;

extern "C" {

size_t mpmw_surrogate_workspace_bytes(int64_t n) { return mpmw::surrogate_workspace_bytes(n); }

int mpmw_stress_surrogate(const mpmw_particles_t *p, const mpmw_params_t *prm, const void *packed,
                          const float *mlp_params, float gate_tol, int audit_per_mille, uint64_t audit_seed,
                          uint32_t *stats, uint32_t *status, void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    if (!p || !prm || !packed || !mlp_params || !stats) { set_error("stress_surrogate: NULL argument"); return MPMW_E_ARG; }
    if (p->n < 0) { set_error("stress_surrogate: negative particle count"); return MPMW_E_ARG; }
    if (count_too_large(p->n, "stress_surrogate")) return MPMW_E_ARG;
    if (p->n == 0) return MPMW_OK;
    if (!p->x || !p->v || !p->C || !p->F || !p->F_trial || !p->stress || !p->active || !p->material || !p->mu ||
        !p->lam || !p->ys || !p->alpha || !p->damage || !p->acc_strain || !p->strain_criteria || !p->hardening ||
        !p->softening || !p->eta_shear || !p->eta_bulk || !p->density || !p->x_pc || !p->v_pc) {
        set_error("stress_surrogate: a required particle array is NULL");
        return MPMW_E_ARG;
    }
    if (!workspace || ws_bytes < surrogate_workspace_bytes(p->n)) {
        set_error("stress_surrogate: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  surrogate_workspace_bytes(p->n));
        return MPMW_E_WORKSPACE;
    }
    cudaStream_t s = as_stream(stream);
    SurrWork W = carve(workspace, p->n);
    if (cudaMemsetAsync(W.count, 0, sizeof(int), s) != cudaSuccess) { set_error("stress_surrogate: memset failed"); return MPMW_E_DEVICE; }
    k_surr_classify<<<grid_for(p->n), kBlock, 0, s>>>(*p, prm->eff, W);
    MPMW_TRY_LAUNCH("k_surr_classify");
    int rc = launch_mlp_infer_tc_dev(packed, mlp_params, W.feat, p->n, W.count, W.out, status, s);
    if (rc != MPMW_OK) return rc;
    k_surr_finish<<<148 * 8, kBlock, 0, s>>>(*p, prm->eff, W, gate_tol, audit_per_mille, audit_seed, stats);
    return check_launch("k_surr_finish");
}

}  // extern "C"
