// mpmw_math.cuh -- per-particle device math of the MPM substep.
//
// Compiled with -fmad=false: every expression below rounds once per operator,
// left to right, so results are reproducible operation by operation.  The
// SVD is our own (cyclic Jacobi on F^T F + Gram-Schmidt QR of F V); it stands
// in for wp.svd3 used by the reference at utils/mpmRoutines.py:288,339.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mpmw {

__device__ __forceinline__ float rmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float rmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float dot3(const float *a, const float *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
__device__ __forceinline__ float len3(const float *a) { return sqrtf(dot3(a, a)); }

// wp.normalize: zero vector -> zero, otherwise component-wise division
__device__ __forceinline__ void normalize3(const float *a, float *o)
{
    float l = len3(a);
    if (l > 0.f) { o[0] = a[0] / l; o[1] = a[1] / l; o[2] = a[2] / l; }
    else { o[0] = o[1] = o[2] = 0.f; }
}

// C = A B, entries ((a0 b0 + a1 b1) + a2 b2)
__device__ __forceinline__ void matmul3(const float *A, const float *B, float *C)
{
    float T[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            T[3 * r + c] = (A[3 * r + 0] * B[0 + c] + A[3 * r + 1] * B[3 + c]) + A[3 * r + 2] * B[6 + c];
#pragma unroll
    for (int k = 0; k < 9; ++k) C[k] = T[k];
}
// C = A B^T
__device__ __forceinline__ void matmul3_bt(const float *A, const float *B, float *C)
{
    float T[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            T[3 * r + c] = (A[3 * r + 0] * B[3 * c + 0] + A[3 * r + 1] * B[3 * c + 1]) + A[3 * r + 2] * B[3 * c + 2];
#pragma unroll
    for (int k = 0; k < 9; ++k) C[k] = T[k];
}

// ---------------------------------------------------------------------------
// 3x3 SVD: F = U diag(s) V^T, U and V proper rotations, s0 >= s1 >= |s2|,
// sign(s2) = sign(det F).
// ---------------------------------------------------------------------------
constexpr int kSvdMaxSweeps = 6;

__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// One Jacobi rotation zeroing S[P][Q] (Golub & Van Loan sec. 8.5, with
// t = 2 a_pq sgn(d) / (|d| + sqrt(d^2 + 4 a_pq^2)), d = a_qq - a_pp, sgn(0) = +1).
// A pair counts as converged when a_pq^2 <= 1e-16 |a_pp a_qq|; returns whether
// it rotated.
template <int P, int Q>
__device__ __forceinline__ bool jacobi_rot(float *S, float *V)
{
    float apq = S[3 * P + Q];
    float app = S[3 * P + P], aqq = S[3 * Q + Q];
    if (apq * apq <= 1e-16f * fabsf(app * aqq)) return false;
    float d = aqq - app;
    float two_apq = 2.f * apq;
    float t = (d < 0.f ? -two_apq : two_apq) / (fabsf(d) + sqrtf(fma_(d, d, two_apq * two_apq)));
    float c = 1.f / sqrtf(fma_(t, t, 1.f));
    float s = t * c;
    S[3 * P + P] = fma_(-t, apq, app);
    S[3 * Q + Q] = fma_(t, apq, aqq);
    S[3 * P + Q] = 0.f;
    S[3 * Q + P] = 0.f;
    constexpr int Rr = 3 - P - Q;
    float srp = S[3 * Rr + P], srq = S[3 * Rr + Q];
    float nrp = fma_(c, srp, -s * srq);
    float nrq = fma_(s, srp, c * srq);
    S[3 * Rr + P] = nrp; S[3 * P + Rr] = nrp;
    S[3 * Rr + Q] = nrq; S[3 * Q + Rr] = nrq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float vkp = V[3 * k + P], vkq = V[3 * k + Q];
        V[3 * k + P] = fma_(c, vkp, -s * vkq);
        V[3 * k + Q] = fma_(s, vkp, c * vkq);
    }
    return true;
}

template <int A, int B>
__device__ __forceinline__ void sort_cols(float *lam, float *V)
{
    if (lam[A] < lam[B]) {
        float t = lam[A]; lam[A] = lam[B]; lam[B] = t;
#pragma unroll
        for (int k = 0; k < 3; ++k) { float u = V[3 * k + A]; V[3 * k + A] = V[3 * k + B]; V[3 * k + B] = u; }
    }
}

// Eigen-decomposition of a symmetric 3x3 A (row-major, full): A = Q diag(lam) Q^T,
// lam in decreasing order, Q a rotation (cyclic Jacobi, as in svd3).
__device__ __forceinline__ void sym_eigen3(const float *A, float *lam, float *Q)
{
    float S[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) S[k] = A[k];
#pragma unroll
    for (int k = 0; k < 9; ++k) Q[k] = 0.f;
    Q[0] = Q[4] = Q[8] = 1.f;
#pragma unroll 1
    for (int sw = 0; sw < kSvdMaxSweeps; ++sw) {
        bool r0 = jacobi_rot<0, 1>(S, Q);
        bool r1 = jacobi_rot<0, 2>(S, Q);
        bool r2 = jacobi_rot<1, 2>(S, Q);
        if (!(r0 || r1 || r2)) break;
    }
    lam[0] = S[0]; lam[1] = S[4]; lam[2] = S[8];
    sort_cols<0, 1>(lam, Q);
    sort_cols<0, 2>(lam, Q);
    sort_cols<1, 2>(lam, Q);
    float detQ = (Q[0] * (Q[4] * Q[8] - Q[5] * Q[7]) - Q[1] * (Q[3] * Q[8] - Q[5] * Q[6])) + Q[2] * (Q[3] * Q[7] - Q[4] * Q[6]);
    if (detQ < 0.f) { Q[2] = -Q[2]; Q[5] = -Q[5]; Q[8] = -Q[8]; }
}

__device__ __forceinline__ void svd3(const float *F, float *U, float *sig, float *V)
{
    float S[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            float v = (F[0 + i] * F[0 + j] + F[3 + i] * F[3 + j]) + F[6 + i] * F[6 + j];
            S[3 * i + j] = v; S[3 * j + i] = v;
        }
#pragma unroll
    for (int k = 0; k < 9; ++k) V[k] = 0.f;
    V[0] = V[4] = V[8] = 1.f;
#pragma unroll 1
    for (int sw = 0; sw < kSvdMaxSweeps; ++sw) {
        bool r0 = jacobi_rot<0, 1>(S, V);
        bool r1 = jacobi_rot<0, 2>(S, V);
        bool r2 = jacobi_rot<1, 2>(S, V);
        if (!(r0 || r1 || r2)) break;
    }
    float lam[3] = {S[0], S[4], S[8]};
    sort_cols<0, 1>(lam, V);
    sort_cols<0, 2>(lam, V);
    sort_cols<1, 2>(lam, V);
    float detV = (V[0] * (V[4] * V[8] - V[5] * V[7]) - V[1] * (V[3] * V[8] - V[5] * V[6])) + V[2] * (V[3] * V[7] - V[4] * V[6]);
    if (detV < 0.f) { V[2] = -V[2]; V[5] = -V[5]; V[8] = -V[8]; }
    float B[9];
    matmul3(F, V, B);
    float b0[3] = {B[0], B[3], B[6]}, b1[3] = {B[1], B[4], B[7]}, b2[3] = {B[2], B[5], B[8]};
    float u0[3], u1[3], u2[3];
    float n0 = len3(b0);
    if (n0 > 1e-30f) { float inv = 1.f / n0; u0[0] = b0[0] * inv; u0[1] = b0[1] * inv; u0[2] = b0[2] * inv; }
    else { u0[0] = 1.f; u0[1] = 0.f; u0[2] = 0.f; n0 = 0.f; }
    float d01 = dot3(u0, b1);
    float w[3] = {b1[0] - d01 * u0[0], b1[1] - d01 * u0[1], b1[2] - d01 * u0[2]};
    float n1 = len3(w);
    if (n1 > 1e-30f) { float inv = 1.f / n1; u1[0] = w[0] * inv; u1[1] = w[1] * inv; u1[2] = w[2] * inv; }
    else {
        float e[3] = {0.f, 0.f, 0.f};
        if (fabsf(u0[0]) < 0.5f) e[0] = 1.f; else e[1] = 1.f;
        float de = dot3(u0, e);
        float g[3] = {e[0] - de * u0[0], e[1] - de * u0[1], e[2] - de * u0[2]};
        float ng = len3(g), inv = 1.f / ng;
        u1[0] = g[0] * inv; u1[1] = g[1] * inv; u1[2] = g[2] * inv;
        n1 = 0.f;
    }
    u2[0] = u0[1] * u1[2] - u0[2] * u1[1];
    u2[1] = u0[2] * u1[0] - u0[0] * u1[2];
    u2[2] = u0[0] * u1[1] - u0[1] * u1[0];
    sig[0] = n0; sig[1] = n1; sig[2] = dot3(u2, b2);
    U[0] = u0[0]; U[3] = u0[1]; U[6] = u0[2];
    U[1] = u1[0]; U[4] = u1[1]; U[7] = u1[2];
    U[2] = u2[0]; U[5] = u2[1]; U[8] = u2[2];
}

// utils/mpmRoutines.py:456-471 kirchoff_stress: tau = U diag(c) V^T F^T
__device__ __forceinline__ void kirchhoff(const float *F, const float *U, const float *V, const float *sig,
                                          float mu, float lam, float *tau)
{
    float s0 = rmax(sig[0], 1e-6f), s1 = rmax(sig[1], 1e-6f), s2 = rmax(sig[2], 1e-6f);
    float l0 = logf(s0), l1 = logf(s1), l2 = logf(s2);
    float lss = (l0 + l1) + l2;
    float c0 = ((2.f * mu) * l0) * (1.f / s0) + (lam * lss) * (1.f / s0);
    float c1 = ((2.f * mu) * l1) * (1.f / s1) + (lam * lss) * (1.f / s1);
    float c2 = ((2.f * mu) * l2) * (1.f / s2) + (lam * lss) * (1.f / s2);
    float UD[9];
#pragma unroll
    for (int r = 0; r < 3; ++r) { UD[3 * r + 0] = U[3 * r + 0] * c0; UD[3 * r + 1] = U[3 * r + 1] * c1; UD[3 * r + 2] = U[3 * r + 2] * c2; }
    float T[9];
    matmul3_bt(UD, V, T);
    matmul3_bt(T, F, tau);
}

// ---------------------------------------------------------------------------
// quadratic B-spline weights (utils/mpmRoutines.py:514-529, 474-483)
// ---------------------------------------------------------------------------
struct Weights {
    int base[3];
    float fx[3];
    float w[3][3];
    float dw[3][3];
};

__device__ __forceinline__ void weights(const float *xp, const float *minb, float inv_dx, Weights &W)
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float gp = (xp[a] - minb[a]) * inv_dx;
        int b = (int)(gp - 0.5f);               // truncation toward zero (wp.int)
        float fx = gp - (float)b;
        float wa = 1.5f - fx, wb = fx - 1.f, wc = fx - 0.5f;
        W.base[a] = b; W.fx[a] = fx;
        W.w[a][0] = (wa * wa) * 0.5f;
        W.w[a][1] = (0.f - wb * wb) + 0.75f;
        W.w[a][2] = (wc * wc) * 0.5f;
        W.dw[a][0] = fx - 1.5f;
        W.dw[a][1] = -2.f * (fx - 1.f);
        W.dw[a][2] = fx - 0.5f;
    }
}

}  // namespace mpmw
