// mpmw_stress.cuh -- per-particle return map + Kirchhoff + Kelvin-Voigt stress.
//
// Reference: utils/mpmRoutines.py:229-312 (compute_stress_from_F_trial),
// :314-453 (drucker_prager_return_mapping), :456-471 (kirchoff_stress).
//
// Two evaluations of the same mathematics:
//  * SVD path (stress_particle, every particle in MPMW_STRESS_SVD mode):
//    svd3 of F_trial, principal log strains, radial return, F_e = U exp(eps) V^T,
//    second svd3 of F_e for the Kirchhoff stress -- operation for operation as
//    the CPU oracle.
//  * tensor path (small_strain_update, MPMW_STRESS_AUTO when |F F^T - I|_F <= 0.02
//    and det F > 0):
//    the model is isotropic and the return is radial, so every quantity the
//    reference takes from principal values is an invariant of the spatial log
//    strain eps = 1/2 ln(F F^T):
//      p = (2 mu / 3 + lam) tr eps,  sigma_eq = 2 mu |dev eps|,
//      eps_new = eps - f dev eps + vc I  (coaxial with eps),
//      F_e = U exp(eps_new) V^T = exp(eps_new - eps) F = e^vc exp(-f dev eps) F,
//      tau = U diag(2 mu ln s + lam sum ln s) U^T = 2 mu eps_new + lam tr(eps_new) I,
//      u = 1/2 tau : eps.
//    With G = F - I (exact in FP32 near identity), X = F F^T - I = G + G^T + G G^T
//    has no cancellation; ln(I + X) and exp(A) are evaluated by truncated series
//    (error < 1e-9 relative at the 0.02 bound).  No SVD, no near-identity log
//    rounding: the result is within ~1e-7 of the FP64 oracle, where the FP32 SVD
//    path is within ~1e-3 for strains of 1e-4.
#pragma once
#include "mpmw_common.cuh"
#include "mpmw_math.cuh"

namespace mpmw {

// Kelvin-Voigt term added to a symmetric Kirchhoff stress (mpmRoutines.py:294-310):
// out = sym(T) + (2 eta_s) dev(sym C) + eta_b tr(sym C) I
__device__ __forceinline__ void add_viscous(const float *T, const float *Cg, float eta_s, float eta_b, float *out)
{
    float sr[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) sr[3 * r + c] = 0.5f * (Cg[3 * r + c] + Cg[3 * c + r]);
    float vrate = (sr[0] + sr[4]) + sr[8];
    float vr3 = vrate / 3.f;
    float te = 2.f * eta_s;
    float bv = eta_b * vrate;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float sym = (T[3 * r + c] + T[3 * c + r]) / 2.f;
            float dev = sr[3 * r + c] - (r == c ? vr3 : 0.f);
            float visc = te * dev + (r == c ? bv : 0.f);
            out[3 * r + c] = sym + visc;
        }
}

// symmetric 3x3 stored as xx yy zz xy xz yz.  C = A B for commuting symmetric
// A, B (polynomials in the same matrix), so C is symmetric.
__device__ __forceinline__ void sym_mul(const float *A, const float *B, float *C)
{
    C[0] = fma_(A[0], B[0], fma_(A[3], B[3], A[4] * B[4]));
    C[1] = fma_(A[3], B[3], fma_(A[1], B[1], A[5] * B[5]));
    C[2] = fma_(A[4], B[4], fma_(A[5], B[5], A[2] * B[2]));
    C[3] = fma_(A[0], B[3], fma_(A[3], B[1], A[4] * B[5]));
    C[4] = fma_(A[0], B[4], fma_(A[3], B[5], A[4] * B[2]));
    C[5] = fma_(A[3], B[4], fma_(A[1], B[5], A[5] * B[2]));
}

__device__ __forceinline__ void sym_to_full(const float *s, float *T)
{
    T[0] = s[0]; T[1] = s[3]; T[2] = s[4];
    T[3] = s[3]; T[4] = s[1]; T[5] = s[5];
    T[6] = s[4]; T[7] = s[5]; T[8] = s[2];
}

// Frobenius double contraction of two symmetric tensors
__device__ __forceinline__ float sym_ddot(const float *a, const float *b)
{
    return fma_(a[0], b[0], fma_(a[1], b[1], a[2] * b[2])) + 2.f * fma_(a[3], b[3], fma_(a[4], b[4], a[5] * b[5]));
}

// exp(A) for a small symmetric A: Taylor to A^5 in Horner form
__device__ __forceinline__ void sym_exp_small(const float *A, float *E)
{
    float P[6], Q[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) P[e] = A[e] * 0.2f + (e < 3 ? 1.f : 0.f);           // I + A/5
    sym_mul(A, P, Q);
#pragma unroll
    for (int e = 0; e < 6; ++e) Q[e] = Q[e] * 0.25f + (e < 3 ? 1.f : 0.f);          // I + A/4 (I + A/5)
    sym_mul(A, Q, P);
#pragma unroll
    for (int e = 0; e < 6; ++e) P[e] = P[e] * (1.f / 3.f) + (e < 3 ? 1.f : 0.f);
    sym_mul(A, P, Q);
#pragma unroll
    for (int e = 0; e < 6; ++e) Q[e] = Q[e] * 0.5f + (e < 3 ? 1.f : 0.f);
    sym_mul(A, Q, P);
#pragma unroll
    for (int e = 0; e < 6; ++e) E[e] = P[e] + (e < 3 ? 1.f : 0.f);
}

// Tensor-form return map for |F F^T - I|_F <= 0.02 and det F > 0 (see file
// header).  Returns 0, touching nothing, when it does not apply; 1 when done;
// 2 when done and the particle became an XPBD particle (T = 0).
// On success writes Fout, the symmetric Kirchhoff stress T (before the viscous
// term) and the same per-particle side effects as the SVD path.
// Material scalars of one particle read ahead of the return map (optional).
struct MatScalars {
    float mu, lam, ys, alpha, D;
};

template <bool HaveXV>
__device__ __forceinline__ int small_strain_update(const mpmw_particles_t &P, float eff, int64_t p, const float *Ft,
                                                    const float *xr, float *vr, float *Fout, float *T,
                                                    const MatScalars *pre = nullptr)
{
    const int64_t n = P.n;
    float G[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = Ft[k] - ((k & 3) == 0 ? 1.f : 0.f);
    float X[6];
    {
        const int rr[6] = {0, 1, 2, 0, 0, 1}, cc[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const int r = rr[e], c = cc[e];
            X[e] = fma_(G[3 * r + 0], G[3 * c + 0], fma_(G[3 * r + 1], G[3 * c + 1],
                        fma_(G[3 * r + 2], G[3 * c + 2], G[3 * r + c] + G[3 * c + r])));
        }
    }
    if (!(sym_ddot(X, X) <= 4e-4f)) return 0;
    // F F^T near I also holds for a reflection (det F ~ -1); the reference's
    // SVD then has a negative singular value, clamped to 0.01, so a reflected
    // F must take the SVD path.  With F F^T near I, det F is near +-1.
    {
        const float det = Ft[0] * (Ft[4] * Ft[8] - Ft[5] * Ft[7]) - Ft[1] * (Ft[3] * Ft[8] - Ft[5] * Ft[6]) +
                          Ft[2] * (Ft[3] * Ft[7] - Ft[4] * Ft[6]);
        if (!(det > 0.f)) return 0;
    }
    // eps = 1/2 ln(I + X) = 1/2 X (I + X (-1/2 I + X (1/3 I - 1/4 X)))
    float eps[6];
    {
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
    }
    float mu, lam, ys, alpha, D;
    if (pre) { mu = pre->mu; lam = pre->lam; ys = pre->ys; alpha = pre->alpha; D = pre->D; }
    else { mu = P.mu[p]; lam = P.lam[p]; ys = P.ys[p]; alpha = P.alpha[p]; D = P.damage[p]; }
    const float tr = (eps[0] + eps[1]) + eps[2];
    const float mean_eps = tr / 3.f;
    float dev[6] = {eps[0] - mean_eps, eps[1] - mean_eps, eps[2] - mean_eps, eps[3], eps[4], eps[5]};
    const float dev_norm = sqrtf(sym_ddot(dev, dev));
    const float twomu = 2.f * mu;
    const float pst = fma_(twomu / 3.f, tr, lam * tr);
    const float sigma_eq = twomu * dev_norm;
    const float yield_eff = (1.f - D) * (ys - alpha * pst);
    float enew[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) enew[e] = eps[e];
#pragma unroll
    for (int k = 0; k < 9; ++k) Fout[k] = Ft[k];
    if (sigma_eq > yield_eff || ys < 0.f || yield_eff < 0.f) {
        const float edn = dev_norm + 1e-6f;
        const float dgamma = edn - yield_eff / (2.f * mu);
        const float dacc = sqrtf(2.f / 3.f) * dgamma;
        P.acc_strain[p] = P.acc_strain[p] + dacc;
        const float sc = P.strain_criteria[p];
        if (sc > 0.f) D = rmin(1.f, D + dacc / sc);
        else D = 1.f;
        if (ys < 0.f || yield_eff < 0.f) D = 1.f;
        P.damage[p] = D;
        if (D >= 1.f && P.material[p] == 1) {
            // phase transition to an XPBD particle (mpmRoutines.py:379-408)
            P.material[p] = 2;
            float xx[3], vv[3];
            if (HaveXV) {
                store9(P.F_trial, n, p, Ft);
                xx[0] = xr[0]; xx[1] = xr[1]; xx[2] = xr[2]; vv[0] = vr[0]; vv[1] = vr[1]; vv[2] = vr[2];
            } else { load3(P.x, n, p, xx); load3(P.v, n, p, vv); }
            store3(P.x_pc, n, p, xx);
            float tau[6];
            const float ltr = lam * tr;
#pragma unroll
            for (int e = 0; e < 6; ++e) tau[e] = fma_(twomu, eps[e], e < 3 ? ltr : 0.f);
            const float u = 0.5f * sym_ddot(tau, eps);
            const float vexp = sqrtf(((2.f * eff) * u) / P.density[p]);
            float vb[3] = {vv[0] + 1e-12f, vv[1] + 1e-12f, vv[2] + 1e-12f};
            float vd[3];
            normalize3(vb, vd);
            vv[0] = vv[0] + vexp * vd[0]; vv[1] = vv[1] + vexp * vd[1]; vv[2] = vv[2] + vexp * vd[2];
            store3(P.v_pc, n, p, vv);
            if (HaveXV) { vr[0] = vv[0]; vr[1] = vv[1]; vr[2] = vv[2]; }
            else store3(P.v, n, p, vv);
            P.ys[p] = 0.f; P.mu[p] = 0.f; P.lam[p] = 0.f; P.alpha[p] = 0.f;
#pragma unroll
            for (int k = 0; k < 9; ++k) T[k] = 0.f;
            return 2;
        }
        const float f = dgamma / edn;
        const float vc = (0.3f * alpha) * dgamma;
#pragma unroll
        for (int e = 0; e < 6; ++e) enew[e] = fma_(-f, dev[e], eps[e]) + (e < 3 ? vc : 0.f);
        const float dsy = ((2.f * mu) * (P.hardening[p] - P.softening[p])) * dgamma;
        ys = rmax(0.f, ys + dsy);
        P.ys[p] = ys;
        // F_e = e^vc exp(-f dev) F_trial
        float A[6], E[6], Ef[9];
#pragma unroll
        for (int e = 0; e < 6; ++e) A[e] = -f * dev[e];
        sym_exp_small(A, E);
        const float s = expf(vc);
#pragma unroll
        for (int e = 0; e < 6; ++e) E[e] = E[e] * s;
        sym_to_full(E, Ef);
        matmul3(Ef, Ft, Fout);
    }
    const float trn = (enew[0] + enew[1]) + enew[2];
    const float ltr = lam * trn;
    float t6[6];
#pragma unroll
    for (int e = 0; e < 6; ++e) t6[e] = fma_(twomu, enew[e], e < 3 ? ltr : 0.f);
    sym_to_full(t6, T);
    return 1;
}

// Return map + Kirchhoff + Kelvin-Voigt for one particle.
// Ft: trial deformation gradient; Cg: velocity gradient C for the viscous
// term; xr/vr: particle position/velocity in registers when HaveXV (fused into
// G2P), otherwise read from (and the velocity written back to) global memory
// on a phase transition.  Outputs F (returned) and the full symmetric stress.
template <bool HaveXV>
__device__ __forceinline__ void stress_particle(const mpmw_particles_t &P, float eff, int mode, int64_t p,
                                                const float *Ft, const float *Cg, const float *xr, float *vr,
                                                float *Fout, float *out)
{
    const int64_t n = P.n;
    float T[9];
    if (mode == MPMW_STRESS_AUTO && small_strain_update<HaveXV>(P, eff, p, Ft, xr, vr, Fout, T)) {
        add_viscous(T, Cg, P.eta_shear[p], P.eta_bulk[p], out);
        return;
    }
    float mu = P.mu[p], lam = P.lam[p], ys = P.ys[p], alpha = P.alpha[p], D = P.damage[p];
#pragma unroll
    for (int k = 0; k < 9; ++k) Fout[k] = Ft[k];
    float U[9], V[9], so[3];
    svd3(Ft, U, so, V);
    float sg0 = rmax(so[0], 0.01f), sg1 = rmax(so[1], 0.01f), sg2 = rmax(so[2], 0.01f);
    float e[3] = {logf(sg0), logf(sg1), logf(sg2)};
    float tr = (e[0] + e[1]) + e[2];
    float mean_eps = tr / 3.f;
    float ed[3] = {e[0] - mean_eps, e[1] - mean_eps, e[2] - mean_eps};
    float twomu = 2.f * mu;
    float ltr = lam * tr;
    float tau[3] = {twomu * e[0] + ltr, twomu * e[1] + ltr, twomu * e[2] + ltr};
    float pst = ((tau[0] + tau[1]) + tau[2]) / 3.f;
    float td[3] = {tau[0] - pst, tau[1] - pst, tau[2] - pst};
    float sigma_eq = len3(td);
    float yield_eff = (1.f - D) * (ys - alpha * pst);
    bool reuse_svd = true;
    if (sigma_eq > yield_eff || ys < 0.f || yield_eff < 0.f) {
        float edn = len3(ed) + 1e-6f;
        float dgamma = edn - yield_eff / (2.f * mu);
        float dacc = sqrtf(2.f / 3.f) * dgamma;
        P.acc_strain[p] = P.acc_strain[p] + dacc;
        float sc = P.strain_criteria[p];
        if (sc > 0.f) D = rmin(1.f, D + dacc / sc);
        else D = 1.f;
        if (ys < 0.f || yield_eff < 0.f) D = 1.f;
        P.damage[p] = D;
        if (D >= 1.f && P.material[p] == 1) {
            // phase transition to an XPBD particle (mpmRoutines.py:379-408)
            P.material[p] = 2;
            float xx[3], vv[3];
            if (HaveXV) {
                // fused into G2P: the reference's G2P wrote this F_trial before the
                // stress phase; the particle now leaves the MPM path, so store it
                store9(P.F_trial, n, p, Ft);
                xx[0] = xr[0]; xx[1] = xr[1]; xx[2] = xr[2]; vv[0] = vr[0]; vv[1] = vr[1]; vv[2] = vr[2];
            } else { load3(P.x, n, p, xx); load3(P.v, n, p, vv); }
            store3(P.x_pc, n, p, xx);
            float rho = P.density[p];
            float u = 0.5f * ((tau[0] * e[0] + tau[1] * e[1]) + tau[2] * e[2]);
            float vexp = sqrtf(((2.f * eff) * u) / rho);
            float vb[3] = {vv[0] + 1e-12f, vv[1] + 1e-12f, vv[2] + 1e-12f};
            float vd[3];
            normalize3(vb, vd);
            vv[0] = vv[0] + vexp * vd[0]; vv[1] = vv[1] + vexp * vd[1]; vv[2] = vv[2] + vexp * vd[2];
            store3(P.v_pc, n, p, vv);
            if (HaveXV) { vr[0] = vv[0]; vr[1] = vv[1]; vr[2] = vv[2]; }
            else store3(P.v, n, p, vv);
            P.ys[p] = 0.f; P.mu[p] = 0.f; P.lam[p] = 0.f; P.alpha[p] = 0.f;
            mu = 0.f; lam = 0.f;
        } else {
            float f = dgamma / edn;
            float beta = 0.3f * alpha;
            float vc = beta * dgamma;
            float en[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) en[k] = (e[k] - f * ed[k]) + vc;
            float dsy = ((2.f * mu) * (P.hardening[p] - P.softening[p])) * dgamma;
            ys = rmax(0.f, ys + dsy);
            P.ys[p] = ys;
            float ex0 = expf(en[0]), ex1 = expf(en[1]), ex2 = expf(en[2]);
            float UD[9];
#pragma unroll
            for (int r = 0; r < 3; ++r) { UD[3 * r + 0] = U[3 * r + 0] * ex0; UD[3 * r + 1] = U[3 * r + 1] * ex1; UD[3 * r + 2] = U[3 * r + 2] * ex2; }
            matmul3_bt(UD, V, Fout);
            reuse_svd = false;
        }
    }
    // Kirchhoff stress from the returned F (second svd3 at mpmRoutines.py:288;
    // identical to the first when F was returned unchanged)
    if (reuse_svd) {
        kirchhoff(Fout, U, V, so, mu, lam, T);
    } else {
        float U2[9], V2[9], s2[3];
        svd3(Fout, U2, s2, V2);
        kirchhoff(Fout, U2, V2, s2, mu, lam, T);
    }
    add_viscous(T, Cg, P.eta_shear[p], P.eta_bulk[p], out);
}

}  // namespace mpmw
