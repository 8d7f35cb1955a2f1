/*
 * mpm_oracle.c -- CPU restatement of the MPMWarpYDW MPM-XPBD substep kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is compiled by
 * oracle/Makefile into oracle/_build/libmpm_oracle_{f32,f64,f32_omp}.so and is
 * loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 * Nothing in the product (mpmwarpydw_b200/) links, imports or calls it.
 *
 * One source, two precisions: REAL is float (-DORACLE_F32) or double
 * (-DORACLE_F64).  The FP32 build follows the same per-operation order as the
 * CUDA kernels (left-to-right sums, no contraction: built with
 * -ffp-contract=off), so it agrees with them to the last bit except where the
 * GPU reorders floating-point atomics (P2G, cell sums, reductions) or where
 * logf/expf differ by an ulp.  The FP64 build is the precision reference.
 * Pinned: tests/test_oracle_golden.py checks it against golden vectors made by
 * executing the reference's own mpmSimulationStep / xpbdSimulationStep source
 * in float64 under a stand-in for the Warp API (tests/golden/gen_golden.py,
 * tests/golden/fakewarp.py) -- agreement to ~1e-13 with identical labels --
 * and against analytic known answers (tests/test_oracle_known_answers.py).
 *
 * Every function cites the reference kernel it restates (paths are relative to
 * the MPMWarpYDW project root).  Arrays use the reference layout: vec3 = 3
 * contiguous REALs per particle, mat33 = 9 contiguous REALs (row-major) per
 * particle, grid arrays are C-ordered (nx, ny, nz[, 3]) with z fastest.
 *
 * Third-party arithmetic restated here (warp-lang, version not pinned by the
 * reference):  wp.svd3 (replaced by the Jacobi SVD below, a published method:
 * cyclic Jacobi eigen-decomposition of F^T F, Golub & Van Loan, "Matrix
 * Computations", sec. 8.5, followed by a Gram-Schmidt QR of F V), wp.HashGrid
 * (hash_grid_build / hash_grid_query restated from its documented behaviour),
 * wp.normalize (zero vector -> zero), wp.int (truncation toward zero).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#if defined(ORACLE_F64)
typedef double REAL;
#define SQRT sqrt
#define LOG log
#define EXP exp
#define FABS fabs
#define POW pow
#else
typedef float REAL;
#define SQRT sqrtf
#define LOG logf
#define EXP expf
#define FABS fabsf
#define POW powf
#endif

#define R(x) ((REAL)(x))

/* status bits (same meaning as the CUDA library's device status word) */
#define ST_OOB 1   /* a stencil node fell outside the grid: access skipped */

/* ------------------------------------------------------------------------ */
/* small vector / matrix helpers (row-major mat33)                           */
/* ------------------------------------------------------------------------ */
static inline REAL rmax(REAL a, REAL b) { return a > b ? a : b; }
static inline REAL rmin(REAL a, REAL b) { return a < b ? a : b; }
static inline REAL dot3(const REAL *a, const REAL *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
static inline REAL len3(const REAL *a) { return SQRT(dot3(a, a)); }
/* wp.normalize: zero vector maps to zero, otherwise component-wise division */
static inline void normalize3(const REAL *a, REAL *o)
{
    REAL l = len3(a);
    if (l > R(0)) { o[0] = a[0] / l; o[1] = a[1] / l; o[2] = a[2] / l; }
    else { o[0] = o[1] = o[2] = R(0); }
}
/* C = A * B  (each entry ((a0 b0 + a1 b1) + a2 b2)) */
static inline void matmul3(const REAL *A, const REAL *B, REAL *C)
{
    REAL T[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            T[3 * r + c] = (A[3 * r + 0] * B[0 + c] + A[3 * r + 1] * B[3 + c]) + A[3 * r + 2] * B[6 + c];
    memcpy(C, T, sizeof(T));
}
/* C = A * B^T */
static inline void matmul3_bt(const REAL *A, const REAL *B, REAL *C)
{
    REAL T[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            T[3 * r + c] = (A[3 * r + 0] * B[3 * c + 0] + A[3 * r + 1] * B[3 * c + 1]) + A[3 * r + 2] * B[3 * c + 2];
    memcpy(C, T, sizeof(T));
}
/* o = M v */
static inline void matvec3(const REAL *M, const REAL *v, REAL *o)
{
    REAL t0 = (M[0] * v[0] + M[1] * v[1]) + M[2] * v[2];
    REAL t1 = (M[3] * v[0] + M[4] * v[1]) + M[5] * v[2];
    REAL t2 = (M[6] * v[0] + M[7] * v[1]) + M[8] * v[2];
    o[0] = t0; o[1] = t1; o[2] = t2;
}

/* ------------------------------------------------------------------------ */
/* 3x3 SVD (stands in for wp.svd3, used at mpmRoutines.py:288 and :339)       */
/*                                                                          */
/* F = U diag(s) V^T with U, V proper rotations, s0 >= s1 >= |s2| and        */
/* sign(s2) = sign(det F).  Algorithm:                                      */
/*  1. S = F^T F;                                                           */
/*  2. cyclic Jacobi sweeps over (0,1),(0,2),(1,2) (jacobi_rot), at most 6, */
/*     ending after a sweep in which every pair was converged; V            */
/*     accumulates the rotations;                                           */
/*  3. sort eigenvalues descending (compare-swap network (0,1),(0,2),(1,2)),*/
/*     then flip V's last column if det V < 0;                              */
/*  4. B = F V; u0 = b0/|b0|; u1 = Gram-Schmidt(b1)/|.|; u2 = u0 x u1;       */
/*     s0 = |b0|, s1 = |b1 - (u0.b1)u0|, s2 = u2.b2.                          */
/* The CUDA kernels implement the same steps in the same order.             */
/* ------------------------------------------------------------------------ */
#define SVD_MAX_SWEEPS 6

/* fused multiply-add with one rounding (the CUDA kernels use __fmaf_rn at the
 * same places) */
#if defined(ORACLE_F64)
#define FMA(a, b, c) fma((a), (b), (c))
#define JACOBI_TOL2 1e-32   /* converge to double precision */
#else
#define FMA(a, b, c) fmaf((a), (b), (c))
#define JACOBI_TOL2 1e-16f  /* the CUDA kernels' threshold */
#endif

/* one Jacobi rotation zeroing S[p][q]; t = 2 a_pq sgn(d) / (|d| + sqrt(d^2 + 4 a_pq^2)),
 * d = a_qq - a_pp, sgn(0) = +1; converged pair (a_pq^2 <= 1e-16 |a_pp a_qq|)
 * is skipped.  Returns whether it rotated. */
static inline int jacobi_rot(REAL *S, REAL *V, int p, int q)
{
    /* S holds the symmetric matrix in full row-major form */
    REAL apq = S[3 * p + q];
    REAL app = S[3 * p + p], aqq = S[3 * q + q];
    if (apq * apq <= JACOBI_TOL2 * FABS(app * aqq)) return 0;
    REAL d = aqq - app;
    REAL two_apq = R(2) * apq;
    REAL t = (d < R(0) ? -two_apq : two_apq) / (FABS(d) + SQRT(FMA(d, d, two_apq * two_apq)));
    REAL c = R(1) / SQRT(FMA(t, t, R(1)));
    REAL s = t * c;
    S[3 * p + p] = FMA(-t, apq, app);
    S[3 * q + q] = FMA(t, apq, aqq);
    S[3 * p + q] = R(0);
    S[3 * q + p] = R(0);
    int r = 3 - p - q;
    REAL srp = S[3 * r + p], srq = S[3 * r + q];
    REAL nrp = FMA(c, srp, -s * srq);
    REAL nrq = FMA(s, srp, c * srq);
    S[3 * r + p] = nrp; S[3 * p + r] = nrp;
    S[3 * r + q] = nrq; S[3 * q + r] = nrq;
    for (int k = 0; k < 3; ++k) {
        REAL vkp = V[3 * k + p], vkq = V[3 * k + q];
        V[3 * k + p] = FMA(c, vkp, -s * vkq);
        V[3 * k + q] = FMA(s, vkp, c * vkq);
    }
    return 1;
}

static inline void swap_cols(REAL *lam, REAL *V, int a, int b)
{
    if (lam[a] < lam[b]) {
        REAL t = lam[a]; lam[a] = lam[b]; lam[b] = t;
        for (int k = 0; k < 3; ++k) { REAL u = V[3 * k + a]; V[3 * k + a] = V[3 * k + b]; V[3 * k + b] = u; }
    }
}

void orc_svd3(const REAL *F, REAL *U, REAL *sig, REAL *V)
{
    REAL S[9];
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            REAL v = (F[0 + i] * F[0 + j] + F[3 + i] * F[3 + j]) + F[6 + i] * F[6 + j];
            S[3 * i + j] = v; S[3 * j + i] = v;
        }
    for (int k = 0; k < 9; ++k) V[k] = R(0);
    V[0] = V[4] = V[8] = R(1);
    for (int sw = 0; sw < SVD_MAX_SWEEPS; ++sw) {
        int r0 = jacobi_rot(S, V, 0, 1);
        int r1 = jacobi_rot(S, V, 0, 2);
        int r2 = jacobi_rot(S, V, 1, 2);
        if (!(r0 || r1 || r2)) break;
    }
    REAL lam[3] = {S[0], S[4], S[8]};
    swap_cols(lam, V, 0, 1);
    swap_cols(lam, V, 0, 2);
    swap_cols(lam, V, 1, 2);
    REAL detV = (V[0] * (V[4] * V[8] - V[5] * V[7]) - V[1] * (V[3] * V[8] - V[5] * V[6])) + V[2] * (V[3] * V[7] - V[4] * V[6]);
    if (detV < R(0)) { V[2] = -V[2]; V[5] = -V[5]; V[8] = -V[8]; }
    REAL B[9];
    matmul3(F, V, B);
    REAL b0[3] = {B[0], B[3], B[6]}, b1[3] = {B[1], B[4], B[7]}, b2[3] = {B[2], B[5], B[8]};
    REAL u0[3], u1[3], u2[3];
    REAL n0 = len3(b0);
    if (n0 > R(1e-30)) { REAL inv = R(1) / n0; u0[0] = b0[0] * inv; u0[1] = b0[1] * inv; u0[2] = b0[2] * inv; }
    else { u0[0] = R(1); u0[1] = R(0); u0[2] = R(0); n0 = R(0); }
    REAL d01 = dot3(u0, b1);
    REAL w[3] = {b1[0] - d01 * u0[0], b1[1] - d01 * u0[1], b1[2] - d01 * u0[2]};
    REAL n1 = len3(w);
    if (n1 > R(1e-30)) { REAL inv = R(1) / n1; u1[0] = w[0] * inv; u1[1] = w[1] * inv; u1[2] = w[2] * inv; }
    else {
        /* rank-deficient: any unit vector orthogonal to u0 */
        REAL e[3] = {R(0), R(0), R(0)};
        if (FABS(u0[0]) < R(0.5)) e[0] = R(1); else e[1] = R(1);
        REAL de = dot3(u0, e);
        REAL g[3] = {e[0] - de * u0[0], e[1] - de * u0[1], e[2] - de * u0[2]};
        REAL ng = len3(g), inv = R(1) / ng;
        u1[0] = g[0] * inv; u1[1] = g[1] * inv; u1[2] = g[2] * inv;
        n1 = R(0);
    }
    u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
    u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
    u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
    sig[0] = n0; sig[1] = n1; sig[2] = dot3(u2, b2);
    U[0] = u0[0]; U[3] = u0[1]; U[6] = u0[2];
    U[1] = u1[0]; U[4] = u1[1]; U[7] = u1[2];
    U[2] = u2[0]; U[5] = u2[1]; U[8] = u2[2];
}

/* ------------------------------------------------------------------------ */
/* material set-up                                                          */
/* ------------------------------------------------------------------------ */

/* mpmRoutines.py:206-226 compute_mu_lam_bulk_from_E_nu */
void orc_mu_lam_bulk(int64_t n, const REAL *E, const REAL *nu, REAL *mu, REAL *lam, REAL *bulk)
{
    for (int64_t p = 0; p < n; ++p) {
        mu[p] = E[p] / (R(2) * (R(1) + nu[p]));
        lam[p] = (E[p] * nu[p]) / ((R(1) + nu[p]) * (R(1) - R(2) * nu[p]));
        bulk[p] = lam[p] + (R(2) / R(3)) * mu[p];
    }
}

/* mpmRoutines.py:51-124 initialize_geostatic_F */
void orc_geostatic_F(int64_t n, const REAL *x, REAL *F, const REAL *mu, const REAL *lam,
                     const REAL *density, REAL gravity, REAL z_top, REAL K0)
{
    for (int64_t p = 0; p < n; ++p) {
        REAL depth = z_top - x[3 * p + 2];
        REAL sigma_v = (-density[p] * gravity) * depth;
        REAL sigma_h = K0 * sigma_v;
        REAL a11 = R(2) * lam[p] + R(2) * mu[p];
        REAL a12 = lam[p];
        REAL a21 = R(2) * lam[p];
        REAL a22 = lam[p] + R(2) * mu[p];
        REAL det = a11 * a22 - a12 * a21;
        REAL eh, ev;
        if (FABS(det) > R(1e-12)) {
            eh = (sigma_h * a22 - sigma_v * a12) / det;
            ev = (a11 * sigma_v - a21 * sigma_h) / det;
        } else { eh = R(0); ev = R(0); }
        REAL *f = F + 9 * p;
        for (int k = 0; k < 9; ++k) f[k] = R(0);
        f[0] = EXP(eh); f[4] = EXP(eh); f[8] = EXP(ev);
    }
}

/* mpmRoutines.py:127-203 initialize_geostatic_F_planestrain */
void orc_geostatic_F_planestrain(int64_t n, const REAL *x, REAL *F, const REAL *mu, const REAL *lam,
                                 const REAL *density, REAL g, REAL z_top, REAL K0)
{
    for (int64_t p = 0; p < n; ++p) {
        REAL depth = z_top - x[3 * p + 2];
        REAL exx, eyy, ezz;
        if (depth > R(0)) {
            REAL muv = mu[p], lv = lam[p];
            REAL nu = lv / (R(2) * (lv + muv));
            REAL E = (muv * (R(3) * lv + R(2) * muv)) / (lv + muv);
            REAL sv = (-density[p] * g) * depth;
            REAL sh = K0 * sv;
            REAL syy = nu * (sh + sv);
            exx = (sh - nu * (syy + sv)) / E;
            eyy = R(0);
            ezz = (sv - nu * (sh + syy)) / E;
        } else { exx = eyy = ezz = R(0); }
        REAL *f = F + 9 * p;
        for (int k = 0; k < 9; ++k) f[k] = R(0);
        f[0] = EXP(exx); f[4] = EXP(eyy); f[8] = EXP(ezz);
    }
}

/* ------------------------------------------------------------------------ */
/* stress: Drucker-Prager return map + Kirchhoff stress + Kelvin-Voigt       */
/* ------------------------------------------------------------------------ */

/* mpmRoutines.py:456-471 kirchoff_stress; result tau = U diag(c) V^T F^T */
static void kirchhoff(const REAL *F, const REAL *U, const REAL *V, const REAL *sig, REAL mu, REAL lam, REAL *tau)
{
    REAL s0 = rmax(sig[0], R(1e-6)), s1 = rmax(sig[1], R(1e-6)), s2 = rmax(sig[2], R(1e-6));
    REAL l0 = LOG(s0), l1 = LOG(s1), l2 = LOG(s2);
    REAL lss = (l0 + l1) + l2;
    REAL c0 = ((R(2) * mu) * l0) * (R(1) / s0) + (lam * lss) * (R(1) / s0);
    REAL c1 = ((R(2) * mu) * l1) * (R(1) / s1) + (lam * lss) * (R(1) / s1);
    REAL c2 = ((R(2) * mu) * l2) * (R(1) / s2) + (lam * lss) * (R(1) / s2);
    REAL UD[9];
    for (int r = 0; r < 3; ++r) { UD[3 * r + 0] = U[3 * r + 0] * c0; UD[3 * r + 1] = U[3 * r + 1] * c1; UD[3 * r + 2] = U[3 * r + 2] * c2; }
    REAL T[9];
    matmul3_bt(UD, V, T);   /* (U D) V^T */
    matmul3_bt(T, F, tau);  /* ... F^T   */
}

/*
 * mpmRoutines.py:229-312 compute_stress_from_F_trial, with the return map of
 * mpmRoutines.py:314-453 drucker_prager_return_mapping inlined.  All per-particle
 * side effects of the reference (accumulated strain, damage, label, phase-change
 * position/velocity, velocity kick, zeroed ys/mu/lam/alpha) are reproduced.
 * constitutive_model is accepted and ignored, as in the reference.
 */
void orc_compute_stress(int64_t n,
                        const int32_t *activeLabel, int32_t *materialLabel,
                        const REAL *x, REAL *v, REAL *x_pc, REAL *v_pc,
                        REAL *F, const REAL *F_trial,
                        REAL *mu, REAL *lam, REAL *ys, const REAL *hardening, const REAL *softening,
                        const REAL *density, const REAL *strainCriteria, REAL eff,
                        const REAL *eta_shear, const REAL *eta_bulk, const REAL *Cmat, REAL *stress,
                        REAL *acc, REAL *damage, int constitutive_model, REAL *alpha)
{
    (void)constitutive_model;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t p = 0; p < n; ++p) {
        if (!(materialLabel[p] <= 1)) continue;
        if (activeLabel[p] != 1) continue;
        const REAL *Ft = F_trial + 9 * p;
        REAL U[9], V[9], so[3];
        orc_svd3(Ft, U, so, V);
        REAL sg[3] = {rmax(so[0], R(0.01)), rmax(so[1], R(0.01)), rmax(so[2], R(0.01))};
        REAL e[3] = {LOG(sg[0]), LOG(sg[1]), LOG(sg[2])};
        REAL tr = (e[0] + e[1]) + e[2];
        REAL mean_eps = tr / R(3);
        REAL ed[3] = {e[0] - mean_eps, e[1] - mean_eps, e[2] - mean_eps};
        REAL twomu = R(2) * mu[p];
        REAL ltr = lam[p] * tr;
        REAL tau[3] = {twomu * e[0] + ltr, twomu * e[1] + ltr, twomu * e[2] + ltr};
        REAL pst = ((tau[0] + tau[1]) + tau[2]) / R(3);
        REAL td[3] = {tau[0] - pst, tau[1] - pst, tau[2] - pst};
        REAL sigma_eq = len3(td);
        REAL yield_eff = (R(1) - damage[p]) * (ys[p] - alpha[p] * pst);
        REAL Fe[9];
        int use_trial = 1;
        if (sigma_eq > yield_eff || ys[p] < R(0) || yield_eff < R(0)) {
            REAL edn = len3(ed) + R(1e-6);
            REAL dgamma = edn - yield_eff / (R(2) * mu[p]);
            REAL dacc = SQRT(R(2) / R(3)) * dgamma;
            acc[p] += dacc;
            if (strainCriteria[p] > R(0)) damage[p] = rmin(R(1), damage[p] + dacc / strainCriteria[p]);
            else damage[p] = R(1);
            if (ys[p] < R(0) || yield_eff < R(0)) damage[p] = R(1);
            if (damage[p] >= R(1) && materialLabel[p] == 1) {
                materialLabel[p] = 2;
                x_pc[3 * p + 0] = x[3 * p + 0]; x_pc[3 * p + 1] = x[3 * p + 1]; x_pc[3 * p + 2] = x[3 * p + 2];
                REAL rho = density[p];
                REAL u = R(0.5) * ((tau[0] * e[0] + tau[1] * e[1]) + tau[2] * e[2]);
                REAL vexp = SQRT(((R(2) * eff) * u) / rho);
                REAL vv[3] = {v[3 * p + 0] + R(1e-12), v[3 * p + 1] + R(1e-12), v[3 * p + 2] + R(1e-12)};
                REAL vd[3];
                normalize3(vv, vd);
                for (int k = 0; k < 3; ++k) v[3 * p + k] = v[3 * p + k] + vexp * vd[k];
                for (int k = 0; k < 3; ++k) v_pc[3 * p + k] = v[3 * p + k];
                ys[p] = R(0); mu[p] = R(0); lam[p] = R(0); alpha[p] = R(0);
            } else {
                REAL f = dgamma / edn;
                REAL beta = R(0.3) * alpha[p];
                REAL vc = beta * dgamma;
                REAL en[3];
                for (int k = 0; k < 3; ++k) en[k] = (e[k] - f * ed[k]) + vc;
                REAL dsy = ((R(2) * mu[p]) * (hardening[p] - softening[p])) * dgamma;
                ys[p] = rmax(R(0), ys[p] + dsy);
                if (ys[p] < R(0)) { ys[p] = R(0); mu[p] = R(0); lam[p] = R(0); }
                REAL ex[3] = {EXP(en[0]), EXP(en[1]), EXP(en[2])};
                REAL UD[9];
                for (int r = 0; r < 3; ++r) { UD[3 * r + 0] = U[3 * r + 0] * ex[0]; UD[3 * r + 1] = U[3 * r + 1] * ex[1]; UD[3 * r + 2] = U[3 * r + 2] * ex[2]; }
                matmul3_bt(UD, V, Fe);
                use_trial = 0;
            }
        }
        REAL *Fp = F + 9 * p;
        if (use_trial) memcpy(Fp, Ft, 9 * sizeof(REAL));
        else memcpy(Fp, Fe, 9 * sizeof(REAL));
        /* second SVD of the returned F (mpmRoutines.py:288) */
        REAL U2[9], V2[9], s2[3], T[9];
        orc_svd3(Fp, U2, s2, V2);
        kirchhoff(Fp, U2, V2, s2, mu[p], lam[p], T);
        REAL sym[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) sym[3 * r + c] = (T[3 * r + c] + T[3 * c + r]) / R(2);
        /* Kelvin-Voigt viscous stress from the velocity gradient C (mpmRoutines.py:294-310) */
        const REAL *G = Cmat + 9 * p;
        REAL sr[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) sr[3 * r + c] = R(0.5) * (G[3 * r + c] + G[3 * c + r]);
        REAL vr = (sr[0] + sr[4]) + sr[8];
        REAL vr3 = vr / R(3);
        REAL te = R(2) * eta_shear[p];
        REAL bv = eta_bulk[p] * vr;
        REAL *out = stress + 9 * p;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                REAL dev = sr[3 * r + c] - (r == c ? vr3 : R(0));
                REAL visc = te * dev + (r == c ? bv : R(0));
                out[3 * r + c] = sym[3 * r + c] + visc;
            }
    }
}

/* ------------------------------------------------------------------------ */
/* quadratic B-spline weights (mpmRoutines.py:514-529, 733-748, 474-483)     */
/* ------------------------------------------------------------------------ */
typedef struct { int base[3]; REAL fx[3]; REAL w[3][3]; REAL dw[3][3]; } wts_t;

static inline void weights(const REAL *xp, const REAL *minb, REAL inv_dx, wts_t *W)
{
    for (int a = 0; a < 3; ++a) {
        REAL gp = (xp[a] - minb[a]) * inv_dx;
        int b = (int)(gp - R(0.5));               /* wp.int truncates toward zero */
        REAL fx = gp - (REAL)b;
        REAL wa = R(1.5) - fx, wb = fx - R(1), wc = fx - R(0.5);
        W->base[a] = b; W->fx[a] = fx;
        W->w[a][0] = (wa * wa) * R(0.5);
        W->w[a][1] = (R(0) - wb * wb) + R(0.75);
        W->w[a][2] = (wc * wc) * R(0.5);
        W->dw[a][0] = fx - R(1.5);
        W->dw[a][1] = R(-2) * (fx - R(1));
        W->dw[a][2] = fx - R(0.5);
    }
}

static inline int64_t node_index(const int *dims, int ix, int iy, int iz)
{
    if (ix < 0 || iy < 0 || iz < 0 || ix >= dims[0] || iy >= dims[1] || iz >= dims[2]) return -1;
    return ((int64_t)ix * dims[1] + iy) * dims[2] + iz;
}

/* mpmRoutines.py:485-569 p2g_apic_with_stress (sequential scatter, particle order) */
int orc_p2g(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
            const REAL *stress, const REAL *x, const REAL *v, const REAL *Cmat,
            const REAL *vol, const REAL *mass, REAL dx, REAL inv_dx, const REAL *minb,
            REAL rpic, const int *dims, REAL *grid_m, REAL *grid_v_in, REAL dt)
{
    int status = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(| : status)
#endif
    for (int64_t p = 0; p < n; ++p) {
        if (!(activeLabel[p] == 1 && materialLabel[p] <= 1)) continue;
        wts_t W;
        weights(x + 3 * p, minb, inv_dx, &W);
        const REAL *C0 = Cmat + 9 * p;
        REAL Cp[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                Cp[3 * r + c] = (R(1) - rpic) * C0[3 * r + c] + (rpic / R(2)) * (C0[3 * r + c] - C0[3 * c + r]);
        if (rpic < R(-0.001)) for (int k = 0; k < 9; ++k) Cp[k] = R(0);
        REAL Sm[9];
        for (int k = 0; k < 9; ++k) Sm[k] = (-vol[p]) * stress[9 * p + k];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    REAL dpos[3] = {((REAL)i - W.fx[0]) * dx, ((REAL)j - W.fx[1]) * dx, ((REAL)k - W.fx[2]) * dx};
                    REAL weight = (W.w[0][i] * W.w[1][j]) * W.w[2][k];
                    REAL dwt[3] = {((W.dw[0][i] * W.w[1][j]) * W.w[2][k]) * inv_dx,
                                   ((W.w[0][i] * W.dw[1][j]) * W.w[2][k]) * inv_dx,
                                   ((W.w[0][i] * W.w[1][j]) * W.dw[2][k]) * inv_dx};
                    REAL ef[3], cd[3];
                    matvec3(Sm, dwt, ef);
                    matvec3(Cp, dpos, cd);
                    REAL wm = weight * mass[p];
                    REAL add[3];
                    for (int a = 0; a < 3; ++a) add[a] = wm * (v[3 * p + a] + cd[a]) + dt * ef[a];
                    int64_t nd = node_index(dims, W.base[0] + i, W.base[1] + j, W.base[2] + k);
                    if (nd < 0) { status |= ST_OOB; continue; }
#ifdef _OPENMP
#pragma omp atomic
                    grid_v_in[3 * nd + 0] += add[0];
#pragma omp atomic
                    grid_v_in[3 * nd + 1] += add[1];
#pragma omp atomic
                    grid_v_in[3 * nd + 2] += add[2];
#pragma omp atomic
                    grid_m[nd] += wm;
#else
                    grid_v_in[3 * nd + 0] += add[0];
                    grid_v_in[3 * nd + 1] += add[1];
                    grid_v_in[3 * nd + 2] += add[2];
                    grid_m[nd] += wm;
#endif
                }
    }
    return status;
}

/* mpmRoutines.py:690-704 grid_normalization_and_gravity */
void orc_grid_normalize(int64_t G, const REAL *grid_m, const REAL *grid_v_in, REAL *grid_v_out,
                        const REAL *gravity, REAL dt)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t g = 0; g < G; ++g) {
        if (grid_m[g] > R(1e-15)) {
            REAL inv = R(1) / grid_m[g];
            for (int a = 0; a < 3; ++a) grid_v_out[3 * g + a] = grid_v_in[3 * g + a] * inv + dt * gravity[a];
        }
    }
}

/* mpmRoutines.py:706-711 add_damping_via_grid */
void orc_grid_damping(int64_t G, REAL *grid_v_out, REAL scale)
{
    for (int64_t g = 0; g < 3 * G; ++g) grid_v_out[g] = grid_v_out[g] * scale;
}

/* mpmRoutines.py:915-940 apply_coulomb_friction */
static inline REAL coulomb(REAL v, REAL mu, REAL dt, REAL g)
{
    if (FABS(v) < R(1e-12)) return R(0);
    REAL dvf = (mu * g) * dt;
    REAL s = v < R(0) ? R(-1) : R(1);
    return s * rmax(FABS(v) - dvf, R(0));
}

/* boundary-condition kernels; bc: 0 friction (mpmRoutines.py:942-993),
 * 1 friction_gradual (:1263-1362), 2 restitution (:1181-1261),
 * 3 absorbing (:1128-1178), 4 plane_strain_y (:996-1063),
 * 5 plane_strain_y_global (:1066-1125) */
void orc_grid_bc(const int *dims, REAL *gv, int bc, REAL mu, REAL rest, REAL dt, REAL g, int pad)
{
    int nx = dims[0], ny = dims[1], nz = dims[2];
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy)
            for (int iz = 0; iz < nz; ++iz) {
                REAL *o = gv + 3 * (((int64_t)ix * ny + iy) * nz + iz);
                REAL v[3] = {o[0], o[1], o[2]};
                if (bc == 0 || bc == 2) {
                    int dim[3] = {nx, ny, nz}, idx[3] = {ix, iy, iz};
                    for (int a = 0; a < 3; ++a) {
                        int t0 = (a + 1) % 3, t1 = (a + 2) % 3;
                        /* low face then high face of axis a; the reference writes from the
                         * velocity read at kernel entry, so a later face overrides */
                        for (int side = 0; side < 2; ++side) {
                            int hit = side == 0 ? (idx[a] <= pad && v[a] < R(0)) : (idx[a] >= dim[a] - pad && v[a] > R(0));
                            if (!hit) continue;
                            REAL w[3];
                            w[a] = bc == 0 ? R(0) : -rest * v[a];
                            w[t0] = coulomb(v[t0], mu, dt, g);
                            w[t1] = coulomb(v[t1], mu, dt, g);
                            o[0] = w[0]; o[1] = w[1]; o[2] = w[2];
                        }
                    }
                } else if (bc == 1) {
                    REAL padf = (REAL)pad;
                    int dim[3] = {nx, ny, nz}, idx[3] = {ix, iy, iz};
                    for (int a = 0; a < 3; ++a) {
                        int t0 = (a + 1) % 3, t1 = (a + 2) % 3;
                        REAL fade; int hit = 0;
                        if (idx[a] < pad && v[a] < R(0)) { fade = (REAL)idx[a] / padf; hit = 1; }
                        else if (idx[a] >= dim[a] - pad && v[a] > R(0)) { fade = (REAL)(dim[a] - 1 - idx[a]) / padf; hit = 1; }
                        if (!hit) continue;
                        REAL fm = mu * (R(1) - fade);
                        REAL w[3];
                        w[t0] = coulomb(v[t0], fm, dt, g);
                        w[t1] = coulomb(v[t1], fm, dt, g);
                        w[a] = R(0) * (R(1) - fade) + v[a] * fade;
                        o[0] = w[0]; o[1] = w[1]; o[2] = w[2];
                    }
                } else if (bc == 3) {
                    REAL padf = (REAL)pad;
                    int dim[3] = {nx, ny, nz}, idx[3] = {ix, iy, iz};
                    for (int a = 0; a < 3; ++a) {
                        for (int side = 0; side < 2; ++side) {
                            int hit = side == 0 ? (idx[a] < 3) : (idx[a] >= dim[a] - 3);
                            if (!hit) continue;
                            REAL lf = side == 0 ? (padf - (REAL)idx[a]) / padf : (padf - (REAL)(dim[a] - 1 - idx[a])) / padf;
                            REAL damp = R(0) * lf + R(1) * (R(1) - lf);
                            o[0] = v[0] * damp; o[1] = v[1] * damp; o[2] = v[2] * damp;
                        }
                    }
                } else if (bc == 4) {
                    /* x faces: friction from the entry velocity */
                    if (ix <= pad && v[0] < R(0)) { o[0] = R(0); o[1] = coulomb(v[1], mu, dt, g); o[2] = coulomb(v[2], mu, dt, g); }
                    if (ix >= nx - pad && v[0] > R(0)) { o[0] = R(0); o[1] = coulomb(v[1], mu, dt, g); o[2] = coulomb(v[2], mu, dt, g); }
                    /* y faces: re-read, zero v_y */
                    if (iy <= pad) { v[0] = o[0]; v[1] = o[1]; v[2] = o[2]; o[0] = v[0]; o[1] = R(0); o[2] = v[2]; }
                    if (iy >= ny - pad) { v[0] = o[0]; v[1] = o[1]; v[2] = o[2]; o[0] = v[0]; o[1] = R(0); o[2] = v[2]; }
                    /* z faces use the (possibly re-read) v */
                    if (iz <= pad && v[2] < R(0)) { REAL a0 = coulomb(v[0], mu, dt, g), a1 = coulomb(v[1], mu, dt, g); o[0] = a0; o[1] = a1; o[2] = R(0); }
                    if (iz >= nz - pad && v[2] > R(0)) { REAL a0 = coulomb(v[0], mu, dt, g), a1 = coulomb(v[1], mu, dt, g); o[0] = a0; o[1] = a1; o[2] = R(0); }
                } else if (bc == 5) {
                    o[1] = R(0);
                    v[0] = o[0]; v[1] = o[1]; v[2] = o[2];
                    if (ix <= pad && v[0] < R(0)) { o[0] = R(0); o[1] = R(0); o[2] = coulomb(v[2], mu, dt, g); }
                    if (ix >= nx - pad && v[0] > R(0)) { o[0] = R(0); o[1] = R(0); o[2] = coulomb(v[2], mu, dt, g); }
                    if (iz <= pad && v[2] < R(0)) { o[0] = coulomb(v[0], mu, dt, g); o[1] = R(0); o[2] = R(0); }
                    if (iz >= nz - pad && v[2] > R(0)) { o[0] = coulomb(v[0], mu, dt, g); o[1] = R(0); o[2] = R(0); }
                }
            }
}

/* mpmRoutines.py:715-776 g2p and :779-802 update_cov */
int orc_g2p(int64_t n, REAL dt, const int32_t *activeLabel, const int32_t *materialLabel,
            REAL *x, REAL *v, REAL *Cmat, const REAL *F, REAL *F_trial, REAL *cov,
            REAL inv_dx, const int *dims, const REAL *grid_v_out, int update_cov, const REAL *minb)
{
    int status = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(| : status)
#endif
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1) continue;
        if (!(materialLabel[p] <= 1)) continue;
        wts_t W;
        weights(x + 3 * p, minb, inv_dx, &W);
        REAL nv[3] = {0, 0, 0}, nC[9] = {0}, nF[9] = {0};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                for (int k = 0; k < 3; ++k) {
                    REAL dpos[3] = {(REAL)i - W.fx[0], (REAL)j - W.fx[1], (REAL)k - W.fx[2]};
                    REAL weight = (W.w[0][i] * W.w[1][j]) * W.w[2][k];
                    int64_t nd = node_index(dims, W.base[0] + i, W.base[1] + j, W.base[2] + k);
                    REAL gvv[3] = {0, 0, 0};
                    if (nd < 0) status |= ST_OOB;
                    else { gvv[0] = grid_v_out[3 * nd]; gvv[1] = grid_v_out[3 * nd + 1]; gvv[2] = grid_v_out[3 * nd + 2]; }
                    for (int a = 0; a < 3; ++a) nv[a] = nv[a] + gvv[a] * weight;
                    REAL sc = (weight * inv_dx) * R(4);
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) nC[3 * r + c] = nC[3 * r + c] + (gvv[r] * dpos[c]) * sc;
                    REAL dwt[3] = {((W.dw[0][i] * W.w[1][j]) * W.w[2][k]) * inv_dx,
                                   ((W.w[0][i] * W.dw[1][j]) * W.w[2][k]) * inv_dx,
                                   ((W.w[0][i] * W.w[1][j]) * W.dw[2][k]) * inv_dx};
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) nF[3 * r + c] = nF[3 * r + c] + gvv[r] * dwt[c];
                }
        for (int a = 0; a < 3; ++a) { v[3 * p + a] = nv[a]; x[3 * p + a] = x[3 * p + a] + dt * nv[a]; }
        memcpy(Cmat + 9 * p, nC, sizeof(nC));
        REAL A[9];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) A[3 * r + c] = (r == c ? R(1) : R(0)) + nF[3 * r + c] * dt;
        matmul3(A, F + 9 * p, F_trial + 9 * p);
        if (update_cov) {
            REAL *cv = cov + 6 * p;
            REAL cn[9] = {cv[0], cv[1], cv[2], cv[1], cv[3], cv[4], cv[2], cv[4], cv[5]};
            REAL a1[9], a2[9];
            matmul3(nF, cn, a1);
            matmul3_bt(cn, nF, a2);
            REAL cn1[9];
            for (int k = 0; k < 9; ++k) cn1[k] = cn[k] + dt * (a1[k] + a2[k]);
            cv[0] = cn1[0]; cv[1] = cn1[1]; cv[2] = cn1[2]; cv[3] = cn1[4]; cv[4] = cn1[5]; cv[5] = cn1[8];
        }
    }
    return status;
}

/* mpmRoutines.py:817-856 accumulate_cell_divergence */
int orc_vlc_accumulate(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
                       const REAL *x, const REAL *Cmat, const REAL *vol, REAL inv_dx, const REAL *minb,
                       const int *dims, REAL *cell_div, REAL *cell_vol)
{
    int status = 0;
    for (int64_t p = 0; p < n; ++p) {
        if (!(activeLabel[p] == 1 && materialLabel[p] <= 1)) continue;
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = (int)((x[3 * p + a] - minb[a]) * inv_dx);
        const REAL *G = Cmat + 9 * p;
        REAL div = (G[0] + G[4]) + G[8];
        int64_t nd = node_index(dims, c[0], c[1], c[2]);
        if (nd < 0) { status |= ST_OOB; continue; }
        cell_div[nd] += div * vol[p];
        cell_vol[nd] += vol[p];
    }
    return status;
}

/* mpmRoutines.py:859-911 apply_volumetric_locking_correction */
int orc_vlc_apply(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
                  const REAL *x, REAL *Cmat, REAL inv_dx, const REAL *minb, const int *dims,
                  const REAL *cell_div, const REAL *cell_vol)
{
    int status = 0;
    for (int64_t p = 0; p < n; ++p) {
        if (!(activeLabel[p] == 1 && materialLabel[p] <= 1)) continue;
        int c[3];
        for (int a = 0; a < 3; ++a) c[a] = (int)((x[3 * p + a] - minb[a]) * inv_dx);
        int64_t nd = node_index(dims, c[0], c[1], c[2]);
        REAL vs = R(0), cd = R(0);
        if (nd < 0) status |= ST_OOB;
        else { vs = cell_vol[nd]; cd = cell_div[nd]; }
        REAL dvc = vs > R(1e-20) ? cd / vs : R(0);
        REAL *G = Cmat + 9 * p;
        REAL dvp = (G[0] + G[4]) + G[8];
        REAL corr = (dvc - dvp) / R(3);
        G[0] = G[0] + corr; G[4] = G[4] + corr; G[8] = G[8] + corr;
    }
    return status;
}

/* mpmRoutines.py:1446-1475 deactivate_and_teleport_xpbd_below_datum */
void orc_teleport(int64_t n, REAL *x, REAL *v, int32_t *activeLabel, const int32_t *materialLabel,
                  REAL z_datum, REAL dist)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] == 1 && materialLabel[p] == 2 && x[3 * p + 2] < z_datum) {
            activeLabel[p] = 0;
            x[3 * p + 2] = x[3 * p + 2] - dist;
            v[3 * p] = v[3 * p + 1] = v[3 * p + 2] = R(0);
        }
    }
}

/* mpmRoutines.py:3-21 creep_by_damage_with_baseline */
void orc_creep(int64_t n, const int32_t *materialLabel, const REAL *damage, REAL *ys, const REAL *ys_base,
               REAL dt, REAL base_creep, REAL damage_creep, REAL damage_exponent)
{
    for (int64_t p = 0; p < n; ++p) {
        if (materialLabel[p] > 1) continue;
        REAL rate = base_creep + damage_creep * POW(damage[p], damage_exponent);
        REAL decay = (rate * ys_base[p]) * dt;
        ys[p] = rmax(R(0), ys[p] - decay);
    }
}

/* ------------------------------------------------------------------------ */
/* hash grid (restates wp.HashGrid: simStates.py:174, simulationRoutines.py:311,
 * queried at xpbdRoutines.py:168-182)                                      */
/* cell of a point: truncating casts of p * (1/cell_width), offset by 2^20,  */
/* clamped at 0, reduced modulo the hash dims; hash = z*(dx*dy) + y*dx + x.  */
/* Points are stable-sorted by hash; cell_starts/ends delimit each hash.    */
/* ------------------------------------------------------------------------ */
static inline int hash_index(const int *hd, int x, int y, int z)
{
    const int origin = 1 << 20;
    x += origin; y += origin; z += origin;
    if (x < 0) x = 0;
    if (y < 0) y = 0;
    if (z < 0) z = 0;
    int cx = x % hd[0], cy = y % hd[1], cz = z % hd[2];
    return cz * (hd[0] * hd[1]) + cy * hd[0] + cx;
}

/* point_ids[n] (sorted order), cell_starts/cell_ends[hd0*hd1*hd2], point_cells[n] (hash per point, input order) */
void orc_hash_build(int64_t n, const float *x, float cell_width, const int *hd,
                    int32_t *point_cells, int32_t *point_ids, int32_t *cell_starts, int32_t *cell_ends)
{
    float inv = 1.0f / cell_width;
    int ncell = hd[0] * hd[1] * hd[2];
    for (int64_t p = 0; p < n; ++p) {
        int cx = (int)(x[3 * p + 0] * inv), cy = (int)(x[3 * p + 1] * inv), cz = (int)(x[3 * p + 2] * inv);
        point_cells[p] = hash_index(hd, cx, cy, cz);
    }
    /* stable counting sort */
    int32_t *cnt = (int32_t *)calloc((size_t)ncell + 1, sizeof(int32_t));
    for (int64_t p = 0; p < n; ++p) cnt[point_cells[p] + 1]++;
    for (int c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
    for (int c = 0; c < ncell; ++c) { cell_starts[c] = 0; cell_ends[c] = 0; }
    for (int c = 0; c < ncell; ++c) if (cnt[c + 1] > cnt[c]) { cell_starts[c] = cnt[c]; cell_ends[c] = cnt[c + 1]; }
    for (int64_t p = 0; p < n; ++p) point_ids[cnt[point_cells[p]]++] = (int32_t)p;
    free(cnt);
}

typedef struct {
    int xs, ys, zs, xe, ye, ze, x, y, z;
    int ci, ce;
} hquery_t;

static inline void hash_query_begin(hquery_t *q, const int *hd, const int32_t *cs, const int32_t *ce,
                                    const float *pos, float radius, float inv)
{
    q->xs = (int)((pos[0] - radius) * inv);
    q->ys = (int)((pos[1] - radius) * inv);
    q->zs = (int)((pos[2] - radius) * inv);
    int xe = (int)((pos[0] + radius) * inv), ye = (int)((pos[1] + radius) * inv), ze = (int)((pos[2] + radius) * inv);
    q->xe = xe < q->xs + hd[0] - 1 ? xe : q->xs + hd[0] - 1;
    q->ye = ye < q->ys + hd[1] - 1 ? ye : q->ys + hd[1] - 1;
    q->ze = ze < q->zs + hd[2] - 1 ? ze : q->zs + hd[2] - 1;
    q->x = q->xs; q->y = q->ys; q->z = q->zs;
    int c = hash_index(hd, q->x, q->y, q->z);
    q->ci = cs[c]; q->ce = ce[c];
}

static inline int hash_query_next(hquery_t *q, const int *hd, const int32_t *cs, const int32_t *ce,
                                  const int32_t *ids, int *index)
{
    for (;;) {
        if (q->ci < q->ce) { *index = ids[q->ci++]; return 1; }
        q->x++;
        if (q->x > q->xe) { q->x = q->xs; q->y++; }
        if (q->y > q->ye) { q->y = q->ys; q->z++; }
        if (q->z > q->ze) return 0;
        int c = hash_index(hd, q->x, q->y, q->z);
        q->ci = cs[c]; q->ce = ce[c];
    }
}

/* ------------------------------------------------------------------------ */
/* XPBD kernels (xpbdRoutines.py).  The XPBD path is FP32-only in the       */
/* reference (hash grid positions are float); these use REAL like the rest. */
/* ------------------------------------------------------------------------ */

/* xpbdRoutines.py:3-21 reset_mpm_contact_labels */
void orc_reset_labels(int64_t n, const int32_t *activeLabel, int32_t *materialLabel)
{
    for (int64_t p = 0; p < n; ++p) if (activeLabel[p] == 1 && materialLabel[p] == 0) materialLabel[p] = 1;
}

/* xpbdRoutines.py:23-48 integrateParticlesXPBD (in place on x, v) */
void orc_integrate_xpbd(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
                        REAL *x, REAL *v, const REAL *gravity, REAL dt, REAL vmax)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1 || materialLabel[p] != 2) continue;
        REAL v1[3] = {v[3 * p] + gravity[0] * dt, v[3 * p + 1] + gravity[1] * dt, v[3 * p + 2] + gravity[2] * dt};
        REAL m = len3(v1);
        if (m > vmax) { REAL s = vmax / m; v1[0] = v1[0] * s; v1[1] = v1[1] * s; v1[2] = v1[2] * s; }
        for (int a = 0; a < 3; ++a) { x[3 * p + a] = x[3 * p + a] + v1[a] * dt; v[3 * p + a] = v1[a]; }
    }
}

/* xpbdRoutines.py:49-136 my_solve_particle_bound_contacts */
void orc_bound_contacts(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
                        const REAL *x, const REAL *v, const REAL *mass, const REAL *radius,
                        REAL mu, REAL thr, REAL static_mu, const REAL *bmin, const REAL *bmax,
                        REAL dt, REAL relax, REAL *delta)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1) continue;
        if (materialLabel[p] != 2) continue;
        if (mass[p] == R(0)) continue;
        REAL wi = R(1) / mass[p];
        const REAL *xp = x + 3 * p, *vp = v + 3 * p;
        REAL r = radius[p];
        for (int i = 0; i < 3; ++i) {
            for (int side = 0; side < 2; ++side) {
                REAL nrm[3] = {0, 0, 0};
                nrm[i] = side == 0 ? R(1) : R(-1);
                const REAL *b = side == 0 ? bmin : bmax;
                REAL d[3] = {xp[0] - b[0], xp[1] - b[1], xp[2] - b[2]};
                REAL c = rmin(dot3(nrm, d) - r, R(0));
                if (!(c < R(0))) continue;
                REAL ln = c;
                REAL dn[3] = {nrm[0] * ln, nrm[1] * ln, nrm[2] * ln};
                REAL vn = dot3(nrm, vp);
                REAL fmu = mu;
                if (FABS(vn) < thr * r) fmu = static_mu;
                REAL vt[3] = {vp[0] - nrm[0] * vn, vp[1] - nrm[1] * vn, vp[2] - nrm[2] * vn};
                REAL vtl = len3(vt);
                REAL lf = rmax(fmu * ln, -vtl * dt);
                REAL df[3] = {0, 0, 0};
                if (vtl > R(1e-8)) { REAL nv[3]; normalize3(vt, nv); df[0] = nv[0] * lf; df[1] = nv[1] * lf; df[2] = nv[2] * lf; }
                for (int a = 0; a < 3; ++a) delta[3 * p + a] += (((df[a] - dn[a]) / wi) * relax) * wi;
            }
        }
    }
}

/* xpbdRoutines.py:138-219 my_solve_particle_particle_contacts.
 * Reproduces the reference's quirks: the outer checks index by the thread id
 * (the sorted position) while the work uses the sorted point i; k_mu, once
 * switched to the static coefficient, stays switched for later neighbours. */
void orc_particle_contacts(int64_t n, const int32_t *activeLabel, int32_t *materialLabel,
                           const int *hd, const int32_t *cs, const int32_t *ce, const int32_t *ids, float cell_width,
                           const REAL *x, const REAL *v, const REAL *mass, const REAL *radius,
                           REAL k_mu_in, REAL thr, REAL static_mu, REAL k_coh, REAL max_radius,
                           REAL dt, REAL relax, int lock, REAL *deltas)
{
    float inv = 1.0f / cell_width;
    for (int64_t tid = 0; tid < n; ++tid) {
        if (activeLabel[tid] != 1) continue;
        if (!(materialLabel[tid] >= 0)) continue;
        int i = ids[tid];
        if (i == -1) continue;
        REAL xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
        REAL vi[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        REAL rad = radius[i];
        if (mass[tid] == R(0)) continue;
        REAL w1 = R(1) / mass[i];
        float qpos[3] = {(float)xi[0], (float)xi[1], (float)xi[2]};
        REAL qr = (rad + max_radius) + k_coh * rad;
        hquery_t q;
        hash_query_begin(&q, hd, cs, ce, qpos, (float)qr, inv);
        int index;
        REAL dl[3] = {0, 0, 0};
        REAL alpha = R(0);
        REAL k_mu = k_mu_in;
        while (hash_query_next(&q, hd, cs, ce, ids, &index)) {
            if (!(activeLabel[index] == 1 && index != i && mass[index] > R(0))) continue;
            if (materialLabel[i] <= 1 && materialLabel[index] <= 1) continue;
            REAL nn[3] = {xi[0] - x[3 * index], xi[1] - x[3 * index + 1], xi[2] - x[3 * index + 2]};
            REAL d = len3(nn);
            REAL err = (d - rad) - radius[index];
            REAL w2 = R(1) / mass[index];
            REAL denom = w1 + w2;
            if (err <= k_coh && denom > R(0)) {
                if (lock == 1) {
                    if (materialLabel[i] <= 1 && materialLabel[index] == 2) materialLabel[i] = 0;
                    if (materialLabel[i] == 2 && materialLabel[index] <= 1) materialLabel[index] = 0;
                }
            }
            if (err <= k_coh && denom > R(0)) {
                REAL nu[3] = {nn[0] / d, nn[1] / d, nn[2] / d};
                REAL vrel[3] = {vi[0] - v[3 * index], vi[1] - v[3 * index + 1], vi[2] - v[3 * index + 2]};
                REAL ln = err / (R(1) + (alpha * dt) * dt);
                REAL dn[3] = {nu[0] * ln, nu[1] * ln, nu[2] * ln};
                REAL vn = dot3(nu, vrel);
                if (FABS(vn) < thr * rad) k_mu = static_mu;
                REAL vt[3] = {vrel[0] - nu[0] * vn, vrel[1] - nu[1] * vn, vrel[2] - nu[2] * vn};
                REAL lf = rmax(k_mu * ln, -len3(vt) * dt);
                REAL nv[3];
                normalize3(vt, nv);
                REAL df[3] = {nv[0] * lf, nv[1] * lf, nv[2] * lf};
                for (int a = 0; a < 3; ++a) dl[a] = dl[a] + ((df[a] - dn[a]) / denom) * w1;
            }
        }
        for (int a = 0; a < 3; ++a) deltas[3 * i + a] += dl[a] * relax;
    }
}

/* xpbdRoutines.py:221-257 my_apply_particle_deltas */
void orc_apply_deltas(int64_t n, const int32_t *activeLabel, const REAL *x_orig, const REAL *x_pred,
                      const REAL *delta, REAL dt, REAL vmax, REAL *x_out, REAL *v_out)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1) continue;
        REAL d[3] = {delta[3 * p], delta[3 * p + 1], delta[3 * p + 2]};
        if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) d[0] = d[1] = d[2] = R(0);
        REAL xn[3], vn[3];
        for (int a = 0; a < 3; ++a) { xn[a] = x_pred[3 * p + a] + d[a]; vn[a] = (xn[a] - x_orig[3 * p + a]) / dt; }
        REAL m = len3(vn);
        if (m > vmax) { REAL s = vmax / m; vn[0] = vn[0] * s; vn[1] = vn[1] * s; vn[2] = vn[2] * s; }
        for (int a = 0; a < 3; ++a) { x_out[3 * p + a] = xn[a]; v_out[3 * p + a] = vn[a]; }
    }
}

/* xpbdRoutines.py:259-310 apply_mpm_contact_impulses */
void orc_mpm_impulses(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel,
                      const REAL *x_orig, const REAL *v_orig, REAL *x_final, REAL dt, REAL vmax,
                      REAL coupling, int xpbd_only, REAL *v_out)
{
    for (int64_t p = 0; p < n; ++p) {
        if (!(activeLabel[p] == 1 && materialLabel[p] <= 1)) continue;
        for (int a = 0; a < 3; ++a) x_final[3 * p + a] = x_orig[3 * p + a];
        if (xpbd_only == 0) {
            REAL vc[3];
            for (int a = 0; a < 3; ++a) vc[a] = v_orig[3 * p + a] + ((x_final[3 * p + a] - x_orig[3 * p + a]) / dt) * coupling;
            REAL m = len3(vc);
            if (m > vmax) { REAL s = vmax / m; vc[0] = vc[0] * s; vc[1] = vc[1] * s; vc[2] = vc[2] * s; }
            for (int a = 0; a < 3; ++a) v_out[3 * p + a] = vc[a];
        }
    }
}

/* xpbdRoutines.py:312-334 sleepParticles; counts[0] += total, counts[1] += sleeping */
void orc_sleep(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel, REAL thr,
               const REAL *radius, const REAL *prev, REAL *after, REAL *dist, REAL dt, int32_t *counts)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1 || materialLabel[p] != 2) continue;
        counts[0] += 1;
        REAL dd[3] = {after[3 * p] - prev[3 * p], after[3 * p + 1] - prev[3 * p + 1], after[3 * p + 2] - prev[3 * p + 2]};
        REAL d = len3(dd);
        if (d / dt < thr * radius[p]) {
            after[3 * p] = prev[3 * p]; after[3 * p + 1] = prev[3 * p + 1]; after[3 * p + 2] = prev[3 * p + 2];
            counts[1] += 1;
        }
        dist[p] = dist[p] + d;
    }
}

/* xpbdRoutines.py:354-375 swellParticlesType2 */
void orc_swell(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel, const REAL *x_init,
               const REAL *x, REAL *radius, REAL factor_in, REAL factor_max_in, const REAL *swellR, const REAL *baseR)
{
    for (int64_t p = 0; p < n; ++p) {
        if (activeLabel[p] != 1 || materialLabel[p] != 2) continue;
        REAL dd[3] = {x[3 * p] - x_init[3 * p], x[3 * p + 1] - x_init[3 * p + 1], x[3 * p + 2] - x_init[3 * p + 2]};
        REAL dxv = len3(dd) * baseR[p];
        REAL factor = factor_in * baseR[p];
        REAL fmax = factor_max_in * baseR[p];
        if (dxv > factor) {
            REAL nr = baseR[p] + ((swellR[p] - baseR[p]) * (dxv - factor)) / (fmax - factor);
            nr = rmin(rmax(nr, radius[p]), swellR[p]);
            radius[p] = nr;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* reductions (simulationRoutines.py:538-675)                                */
/* ------------------------------------------------------------------------ */
/* out[0] = sum |v|/r over active (velocityConvergence), out[1] = active count,
 * out[2] = sum damage over active, out[3..6] = activeMPM, activeXPBD, inactiveMPM, inactiveXPBD */
void orc_stats(int64_t n, const int32_t *activeLabel, const int32_t *materialLabel, const REAL *v,
               const REAL *radius, const REAL *damage, double *out)
{
    REAL res = R(0), dsum = R(0);
    int64_t na = 0, am = 0, ax = 0, im = 0, ix = 0;
    for (int64_t p = 0; p < n; ++p) {
        int act = activeLabel[p] == 1, xp = materialLabel[p] == 2;
        if (act) { res = res + len3(v + 3 * p) / radius[p]; na++; dsum = dsum + damage[p]; }
        if (xp) { if (act) ax++; else ix++; }
        else { if (act) am++; else im++; }
    }
    out[0] = (double)res; out[1] = (double)na; out[2] = (double)dsum;
    out[3] = (double)am; out[4] = (double)ax; out[5] = (double)im; out[6] = (double)ix;
}

int orc_real_bytes(void) { return (int)sizeof(REAL); }
