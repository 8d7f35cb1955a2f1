// mpmw_mlp.cu -- learned surrogate of the Drucker-Prager return map: training
// samples, FP32 training kernels (forward, backward, Adam) and tensor-core
// inference (tcgen05.mma, BF16 operands, FP32 accumulators in tensor memory).
//
// The return map it learns is the reference's closed-form radial return in
// principal log-strain space (utils/mpmRoutines.py:339-453):
//   tau = 2 mu e + lam tr(e), p = tr(tau)/3, sigma_eq = |dev tau|,
//   yield = (1 - D)(ys - alpha p); plastic if sigma_eq > yield,
//   edn = |dev e| + 1e-6, dgamma = edn - yield / (2 mu), d_acc = sqrt(2/3) dgamma,
//   e_ret = e - (dgamma / edn) dev e + beta dgamma.
// Features and targets are defined in include/mpmw_mlp.h: the targets are the
// return's ratios (ln rho, ln(1 - rho), beta, sqrt(2/3)), so an output error is
// a relative error of the returned deviator and plastic multiplier.
#include <cuda_bf16.h>

#include "mpmw_common.cuh"
#include "mpmw_tma.cuh"
#include "../../include/mpmw_mlp.h"

namespace mpmw {
namespace mlp {

constexpr int IN = MPMW_MLP_IN, H = MPMW_MLP_HID, OUT = MPMW_MLP_OUT, NP = MPMW_MLP_NPARAM;
constexpr int oW1 = 0, oB1 = oW1 + H * IN, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H, oB3 = oW3 + H * H,
              oW4 = oB3 + H, oB4 = oW4 + OUT * H;
static_assert(oB4 + OUT == NP, "parameter packing");

// ---------------------------------------------------------------------------
// samples
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double u01(uint64_t &s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

__device__ __forceinline__ double dp_alpha(double deg)
{
    const double sn = sin(deg * (3.14159265358979323846 / 180.0));
    return 2.0 * sn / (sqrt(3.0) * (3.0 - sn));
}

// Plain principal-space return (double).  Returns 0 for an elastic trial, 1 for
// a plastic return (e_ret, d_acc written), 2 when the reference would set D = 1
// instead (ys < 0 or yield < 0).
__device__ int dp_return(const double *e, double mu, double lam, double ys, double alpha, double beta, double D,
                         double *er, double &dacc)
{
    const double tr = e[0] + e[1] + e[2];
    const double mean = tr / 3.0;
    const double ed[3] = {e[0] - mean, e[1] - mean, e[2] - mean};
    double tau[3], p = 0.0;
    for (int k = 0; k < 3; ++k) { tau[k] = 2.0 * mu * e[k] + lam * tr; p += tau[k]; }
    p /= 3.0;
    double seq = 0.0;
    for (int k = 0; k < 3; ++k) seq += (tau[k] - p) * (tau[k] - p);
    seq = sqrt(seq);
    const double yield_eff = (1.0 - D) * (ys - alpha * p);
    if (ys < 0.0 || yield_eff < 0.0) return 2;
    if (!(seq > yield_eff)) return 0;
    const double edn = sqrt(ed[0] * ed[0] + ed[1] * ed[1] + ed[2] * ed[2]) + 1e-6;
    const double dg = edn - yield_eff / (2.0 * mu);
    dacc = sqrt(2.0 / 3.0) * dg;
    const double f = dg / edn, vc = beta * dg;
    for (int k = 0; k < 3; ++k) er[k] = (e[k] - f * ed[k]) + vc;
    return 1;
}

// smallest ln(1 - rho) kept in a target (trials this close to the yield
// surface are left to the gate's exact fallback)
constexpr double kLn1mRhoMin = -12.0;

__global__ void k_dp_samples(int64_t n, uint64_t seed, float *__restrict__ x, float *__restrict__ y)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double e[3] = {0, 0, 0}, er[3] = {0, 0, 0}, dacc = 0.0, mag = 1e-6, yv = 1.0, alpha = 0, beta = 0, D = 0, nu = 0.25;
    double rho = 0.5;
    for (int attempt = 0; attempt < 64; ++attempt) {
        uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1)) ^ ((uint64_t)attempt << 56);
        mag = pow(10.0, -6.0 + 5.0 * u01(s));
        // direction: normalized Gaussian (Box-Muller)
        double g[3];
        for (int k = 0; k < 3; k += 2) {
            const double u1 = fmax(u01(s), 1e-300), u2 = u01(s);
            const double r = sqrt(-2.0 * log(u1)), th = 6.283185307179586 * u2;
            g[k] = r * cos(th);
            if (k + 1 < 3) g[k + 1] = r * sin(th);
        }
        const double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) + 1e-300;
        for (int k = 0; k < 3; ++k) e[k] = mag * g[k] / gn;
        // sort descending
        if (e[0] < e[1]) { double t = e[0]; e[0] = e[1]; e[1] = t; }
        if (e[1] < e[2]) { double t = e[1]; e[1] = e[2]; e[2] = t; }
        if (e[0] < e[1]) { double t = e[0]; e[0] = e[1]; e[1] = t; }
        alpha = dp_alpha(20.0 + 25.0 * u01(s));
        // half the samples use the reference's fixed dilation beta = 0.3 alpha
        // (utils/mpmRoutines.py:424), half a dilation angle U(0, 10) deg
        beta = u01(s) < 0.5 ? 0.3 * alpha : dp_alpha(10.0 * u01(s));
        const double ys = 1e5 * pow(50.0, u01(s));
        const double E = 1e9 * pow(50.0, u01(s));
        nu = 0.15 + 0.2 * u01(s);
        D = (double)MPMW_SURR_D_MAX * u01(s);
        const double mu = E / (2.0 * (1.0 + nu)), lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        yv = ys / (2.0 * mu);
        if (dp_return(e, mu, lam, ys, alpha, beta, D, er, dacc) == 1) {
            // rho = yield / (2 mu |dev e|), from the same quantities as the return
            const double tr = e[0] + e[1] + e[2], p = (2.0 * mu / 3.0 + lam) * tr;
            const double m3 = tr / 3.0;
            const double nd = sqrt((e[0] - m3) * (e[0] - m3) + (e[1] - m3) * (e[1] - m3) + (e[2] - m3) * (e[2] - m3));
            rho = (1.0 - D) * (ys - alpha * p) / (2.0 * mu * nd);
            if (rho > 0.0 && rho < 1.0) break;
        }
        rho = 0.5;  // (only after 64 elastic attempts)
    }
    float *xo = x + 8 * i, *yo = y + 4 * i;
    xo[0] = (float)(e[0] / mag); xo[1] = (float)(e[1] / mag); xo[2] = (float)(e[2] / mag);
    xo[3] = (float)log10(mag / yv);
    xo[4] = (float)alpha; xo[5] = (float)beta; xo[6] = (float)log1p(-D); xo[7] = (float)nu;
    yo[0] = (float)log(rho);
    yo[1] = (float)fmax(log1p(-rho), kLn1mRhoMin);
    yo[2] = (float)beta;
    yo[3] = (float)sqrt(2.0 / 3.0);
}

// ---------------------------------------------------------------------------
// FP32 training kernels: a CTA holds a tile of kTile samples and all weights
// (rounded to BF16) in shared memory.
// ---------------------------------------------------------------------------
constexpr int kTile = 64;
constexpr int kThreads = 256;
constexpr int kLd = H + 1;  // padded row stride of transposed weights (conflict-free both ways)

struct TrainShared {
    float w1t[IN][kLd], w2t[H][kLd], w3t[H][kLd], w4t[H][OUT + 1];
    float b1[H], b2[H], b3[H], b4[OUT];
    float x[kTile][IN];
    float a1[kTile][H], a2[kTile][H], a3[kTile][H];     // activations
    float d1[kTile][H], d2[kTile][H], d3[kTile][H];     // SiLU'(z)
    float out[kTile][OUT];
    float gz[kTile][H], ga[kTile][H];                   // backward scratch
    float loss;
};

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__device__ __forceinline__ void silu_pair(float z, float &a, float &d)
{
    const float s = 1.f / (1.f + expf(-z));
    a = z * s;
    d = s * (1.f + z * (1.f - s));
}

__device__ void load_weights(TrainShared &S, const float *__restrict__ P)
{
    for (int q = threadIdx.x; q < H * IN; q += blockDim.x) { int j = q / IN, k = q % IN; S.w1t[k][j] = bf16r(P[oW1 + q]); }
    for (int q = threadIdx.x; q < H * H; q += blockDim.x) {
        int j = q / H, k = q % H;
        S.w2t[k][j] = bf16r(P[oW2 + q]);
        S.w3t[k][j] = bf16r(P[oW3 + q]);
    }
    // the last layer stays FP32 (it runs on the CUDA cores at inference)
    for (int q = threadIdx.x; q < OUT * H; q += blockDim.x) { int o = q / H, k = q % H; S.w4t[k][o] = P[oW4 + q]; }
    for (int q = threadIdx.x; q < H; q += blockDim.x) { S.b1[q] = P[oB1 + q]; S.b2[q] = P[oB2 + q]; S.b3[q] = P[oB3 + q]; }
    if (threadIdx.x < OUT) S.b4[threadIdx.x] = P[oB4 + threadIdx.x];
}

// forward over the tile (rows >= rows_valid are zero inputs)
__device__ void tile_forward(TrainShared &S)
{
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, j = q % H;
        float z = S.b1[j];
#pragma unroll
        for (int k = 0; k < IN; ++k) z = fmaf(S.x[s][k], S.w1t[k][j], z);
        silu_pair(z, S.a1[s][j], S.d1[s][j]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, j = q % H;
        float z = S.b2[j];
        for (int k = 0; k < H; ++k) z = fmaf(S.a1[s][k], S.w2t[k][j], z);
        silu_pair(z, S.a2[s][j], S.d2[s][j]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, j = q % H;
        float z = S.b3[j];
        for (int k = 0; k < H; ++k) z = fmaf(S.a2[s][k], S.w3t[k][j], z);
        silu_pair(z, S.a3[s][j], S.d3[s][j]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < kTile * OUT; q += blockDim.x) {
        const int s = q / OUT, o = q % OUT;
        float z = S.b4[o];
        for (int k = 0; k < H; ++k) z = fmaf(S.a3[s][k], S.w4t[k][o], z);
        S.out[s][o] = z;
    }
    __syncthreads();
}

__device__ void load_x(TrainShared &S, const float *__restrict__ X, int64_t row0, int64_t n)
{
    for (int q = threadIdx.x; q < kTile * IN; q += blockDim.x) {
        const int s = q / IN, k = q % IN;
        const int64_t r = row0 + s;
        S.x[s][k] = r < n ? X[r * IN + k] : 0.f;
    }
}

__global__ void __launch_bounds__(kThreads) k_mlp_forward(const float *__restrict__ P, const float *__restrict__ X,
                                                          int64_t n, float *__restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainShared &S = *reinterpret_cast<TrainShared *>(smem_raw);
    const int64_t row0 = (int64_t)blockIdx.x * kTile;
    load_weights(S, P);
    load_x(S, X, row0, n);
    __syncthreads();
    tile_forward(S);
    for (int q = threadIdx.x; q < kTile * OUT; q += blockDim.x) {
        const int s = q / OUT, o = q % OUT;
        if (row0 + s < n) Y[(row0 + s) * OUT + o] = S.out[s][o];
    }
}

// gradient of mean((out - y)^2) over all n*OUT entries
__global__ void __launch_bounds__(kThreads) k_mlp_grad(const float *__restrict__ P, const float *__restrict__ X,
                                                       const float *__restrict__ Yt, int64_t n, float *__restrict__ G,
                                                       float *__restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainShared &S = *reinterpret_cast<TrainShared *>(smem_raw);
    const int64_t row0 = (int64_t)blockIdx.x * kTile;
    const int rows = n - row0 < (int64_t)kTile ? (int)(n - row0) : kTile;
    load_weights(S, P);
    load_x(S, X, row0, n);
    if (threadIdx.x == 0) S.loss = 0.f;
    __syncthreads();
    tile_forward(S);
    const float inv = 2.f / (float)((double)n * OUT);
    // d out (stored in gz[:, 0..3])
    float lsum = 0.f;
    for (int q = threadIdx.x; q < kTile * OUT; q += blockDim.x) {
        const int s = q / OUT, o = q % OUT;
        float d = 0.f;
        if (s < rows) {
            const float r = S.out[s][o] - Yt[(row0 + s) * OUT + o];
            lsum += r * r;
            d = inv * r;
        }
        S.gz[s][o] = d;
    }
    atomicAdd(&S.loss, lsum);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(loss, S.loss / (float)((double)n * OUT));
    // layer 4: weights and bias, and d a3
    for (int q = threadIdx.x; q < OUT * H; q += blockDim.x) {
        const int o = q / H, k = q % H;
        float gw = 0.f;
        for (int s = 0; s < kTile; ++s) gw = fmaf(S.gz[s][o], S.a3[s][k], gw);
        atomicAdd(&G[oW4 + q], gw);
    }
    if (threadIdx.x < OUT) {
        float gb = 0.f;
        for (int s = 0; s < kTile; ++s) gb += S.gz[s][threadIdx.x];
        atomicAdd(&G[oB4 + threadIdx.x], gb);
    }
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, k = q % H;
        float da = 0.f;
#pragma unroll
        for (int o = 0; o < OUT; ++o) da = fmaf(S.gz[s][o], S.w4t[k][o], da);
        S.ga[s][k] = da * S.d3[s][k];  // d z3
    }
    __syncthreads();
    // layer 3
    for (int q = threadIdx.x; q < H * H; q += blockDim.x) {
        const int j = q / H, k = q % H;
        float gw = 0.f;
        for (int s = 0; s < kTile; ++s) gw = fmaf(S.ga[s][j], S.a2[s][k], gw);
        atomicAdd(&G[oW3 + q], gw);
    }
    if (threadIdx.x < H) {
        float gb = 0.f;
        for (int s = 0; s < kTile; ++s) gb += S.ga[s][threadIdx.x];
        atomicAdd(&G[oB3 + threadIdx.x], gb);
    }
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, k = q % H;
        float da = 0.f;
        for (int j = 0; j < H; ++j) da = fmaf(S.ga[s][j], S.w3t[k][j], da);
        S.gz[s][k] = da * S.d2[s][k];  // d z2
    }
    __syncthreads();
    // layer 2
    for (int q = threadIdx.x; q < H * H; q += blockDim.x) {
        const int j = q / H, k = q % H;
        float gw = 0.f;
        for (int s = 0; s < kTile; ++s) gw = fmaf(S.gz[s][j], S.a1[s][k], gw);
        atomicAdd(&G[oW2 + q], gw);
    }
    if (threadIdx.x < H) {
        float gb = 0.f;
        for (int s = 0; s < kTile; ++s) gb += S.gz[s][threadIdx.x];
        atomicAdd(&G[oB2 + threadIdx.x], gb);
    }
    for (int q = threadIdx.x; q < kTile * H; q += blockDim.x) {
        const int s = q / H, k = q % H;
        float da = 0.f;
        for (int j = 0; j < H; ++j) da = fmaf(S.gz[s][j], S.w2t[k][j], da);
        S.ga[s][k] = da * S.d1[s][k];  // d z1
    }
    __syncthreads();
    // layer 1
    for (int q = threadIdx.x; q < H * IN; q += blockDim.x) {
        const int j = q / IN, k = q % IN;
        float gw = 0.f;
        for (int s = 0; s < kTile; ++s) gw = fmaf(S.ga[s][j], S.x[s][k], gw);
        atomicAdd(&G[oW1 + q], gw);
    }
    if (threadIdx.x < H) {
        float gb = 0.f;
        for (int s = 0; s < kTile; ++s) gb += S.ga[s][threadIdx.x];
        atomicAdd(&G[oB1 + threadIdx.x], gb);
    }
}

__global__ void k_mlp_adam(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ M,
                           float *__restrict__ V, float lr, float c1, float c2)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= NP) return;
    const float g = G[q];
    const float m = 0.9f * M[q] + 0.1f * g;
    const float v = 0.999f * V[q] + 0.001f * g * g;
    M[q] = m;
    V[q] = v;
    P[q] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

// ---------------------------------------------------------------------------
// tensor-core inference
// ---------------------------------------------------------------------------
// Operand tiles in shared memory use the canonical K-major layout without
// swizzle: 8x8 BF16 core matrices of 128 contiguous bytes (8 rows of 16 bytes);
// the core matrix (row block rb, k block kb) of an R x K tile sits at
// (rb * K/8 + kb) * 128 bytes.  Descriptor: leading (K-direction) byte offset
// 128, stride (row-direction) byte offset K/8 * 128.
constexpr int kTcRows = 128;                 // M of every MMA (one row per thread)
constexpr int kPackW1 = 0, kPackW2 = 2048, kPackW3 = 2048 + 8192, kPackW4 = 2048 + 2 * 8192;
static_assert(kPackW4 + 2048 == MPMW_MLP_PACKED_BYTES, "packed size");

__host__ __device__ __forceinline__ int core_offset(int r, int k, int K)
{
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__global__ void k_mlp_pack(const float *__restrict__ P, __nv_bfloat16 *__restrict__ W)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned char *base = reinterpret_cast<unsigned char *>(W);
    auto put = [&](int off, int r, int k, int K, float v) {
        *reinterpret_cast<__nv_bfloat16 *>(base + off + core_offset(r, k, K)) = __float2bfloat16_rn(v);
    };
    if (q < H * 16) {  // W1: 64 x 16, [W1 | W1]: inputs 0..7 take the features' hi terms, 8..15 their lo terms
        const int r = q / 16, k = q % 16;
        put(kPackW1, r, k, 16, P[oW1 + r * IN + (k & (IN - 1))]);
    }
    if (q < H * H) {
        const int r = q / H, k = q % H;
        put(kPackW2, r, k, H, P[oW2 + q]);
        put(kPackW3, r, k, H, P[oW3 + q]);
    }
    if (q < 16 * H) {  // W4: 16 x 64 (outputs 4..15 zero)
        const int r = q / H, k = q % H;
        put(kPackW4, r, k, H, r < OUT ? P[oW4 + r * H + k] : 0.f);
    }
}

struct TcShared {
    unsigned char w[MPMW_MLP_PACKED_BYTES];   // B operands
    unsigned char a[kTcRows * H * 2];         // A operand: activations, BF16 hi terms
    unsigned char alo[kTcRows * H * 2];       // A operand: activations, BF16 lo terms (a - hi)
    float w4[OUT][H];                         // last layer, FP32
    float bias[3 * H + OUT];
    uint64_t bar;
    uint32_t tmem;
    int timeout;
};

__device__ __forceinline__ uint64_t smem_desc(const void *p, uint32_t lbo, uint32_t sbo)
{
    const uint64_t a = smem_addr(p);
    return ((a & 0x3FFFFull) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t idesc_bf16(int N)
{
    // F32 accumulate, BF16 A and B, both K-major, N/8, M/16 (M = 128)
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t id, int acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 accumulator columns of this thread's row
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// a = hi + lo with hi = bf16(a), lo = bf16(a - hi): the pair carries about
// 16 mantissa bits, and both terms go through the MMA with the same weights
__device__ __forceinline__ void split_bf16(float a0, float a1, __nv_bfloat162 &hi, __nv_bfloat162 &lo)
{
    hi = __floats2bfloat162_rn(a0, a1);
    const float2 h = __bfloat1622float2(hi);
    lo = __floats2bfloat162_rn(a0 - h.x, a1 - h.y);
}

// write this thread's row of 64 activations into the K = 64 A tiles (hi, lo)
__device__ __forceinline__ void put_row64(unsigned char *a, unsigned char *alo, int r, const float *h)
{
#pragma unroll
    for (int kb = 0; kb < 8; ++kb) {
        __nv_bfloat162 v[4], w[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) split_bf16(h[8 * kb + 2 * c], h[8 * kb + 2 * c + 1], v[c], w[c]);
        *reinterpret_cast<uint4 *>(a + core_offset(r, 8 * kb, H)) = *reinterpret_cast<uint4 *>(v);
        *reinterpret_cast<uint4 *>(alo + core_offset(r, 8 * kb, H)) = *reinterpret_cast<uint4 *>(w);
    }
}

// n_dev (optional): a device count that lowers n (a worklist filled by an
// earlier kernel); CTAs past it exit before touching tensor memory.
__global__ void __launch_bounds__(kTcRows) k_mlp_infer_tc(const unsigned char *__restrict__ packed,
                                                          const float *__restrict__ P, const float *__restrict__ X,
                                                          int64_t n, float *__restrict__ Y, uint32_t *status,
                                                          const int *__restrict__ n_dev)
{
    if (n_dev) n = min(n, (int64_t)*n_dev);
    if ((int64_t)blockIdx.x * kTcRows >= n) return;  // uniform
    extern __shared__ __align__(1024) unsigned char smem_tc[];
    TcShared &S = *reinterpret_cast<TcShared *>(smem_tc + ((1024u - (smem_addr(smem_tc) & 1023u)) & 1023u));
    const int t = threadIdx.x, warp = t >> 5;
    const int64_t row = (int64_t)blockIdx.x * kTcRows + t;
    // weights and biases
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(packed);
        uint4 *dst = reinterpret_cast<uint4 *>(S.w);
        for (int q = t; q < MPMW_MLP_PACKED_BYTES / 16; q += kTcRows) dst[q] = src[q];
        for (int q = t; q < H; q += kTcRows) {
            S.bias[q] = P[oB1 + q];
            S.bias[H + q] = P[oB2 + q];
            S.bias[2 * H + q] = P[oB3 + q];
        }
        if (t < OUT) S.bias[3 * H + t] = P[oB4 + t];
        for (int q = t; q < OUT * H; q += kTcRows) S.w4[q / H][q % H] = P[oW4 + q];
    }
    // layer-1 operand: this row's 8 features as hi terms (k 0..7) and lo terms
    // (k 8..15), against [W1 | W1]
    {
        float f[IN];
#pragma unroll
        for (int k = 0; k < IN; ++k) f[k] = row < n ? X[row * IN + k] : 0.f;
        __nv_bfloat162 v[4], w[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) split_bf16(f[2 * c], f[2 * c + 1], v[c], w[c]);
        *reinterpret_cast<uint4 *>(S.a + core_offset(t, 0, 16)) = *reinterpret_cast<uint4 *>(v);
        *reinterpret_cast<uint4 *>(S.a + core_offset(t, 8, 16)) = *reinterpret_cast<uint4 *>(w);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&S.tmem)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) { mbar_init(&S.bar, 1); S.timeout = 0; }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    unsigned phase = 0;
    float h[H];
    // layers 1-3 on the tensor cores (hi and lo operand terms into one
    // accumulator), the last layer in FP32 from the registers
    for (int layer = 0; layer < 3; ++layer) {
        const int K = layer == 0 ? 16 : H;
        const int N = H;
        if (t == 0 && !S.timeout) {
            tc_fence_after();
            const unsigned char *w = S.w + (layer == 0 ? kPackW1 : layer == 1 ? kPackW2 : kPackW3);
            const uint32_t id = idesc_bf16(N);
            const int terms = layer == 0 ? 1 : 2;  // layer 1 holds both terms in its K = 16
            for (int term = 0; term < terms; ++term) {
                const unsigned char *a = term == 0 ? S.a : S.alo;
                for (int kk = 0; kk < K / 16; ++kk) {
                    const uint64_t ad = smem_desc(a + kk * 256, 128, (K / 8) * 128);
                    const uint64_t bd = smem_desc(w + kk * 256, 128, (K / 8) * 128);
                    tc_mma(tmem, ad, bd, id, (term | kk) > 0);
                }
            }
            tc_commit(&S.bar);
        }
        if (!mbar_wait_bounded(&S.bar, phase)) {
            S.timeout = 1;
            raise_status(status, MPMW_ST_TIMEOUT);
        }
        phase ^= 1u;
        tc_fence_after();
        // accumulators of this thread's row
        for (int c = 0; c < N; c += 16) tc_ld16(lane_addr + (uint32_t)c, h + c);
        tc_wait_ld();
        {
            const float *b = S.bias + layer * H;
#pragma unroll
            for (int j = 0; j < H; ++j) {
                const float z = h[j] + b[j];
                h[j] = z / (1.f + expf(-z));
            }
        }
        if (layer < 2) {
            put_row64(S.a, S.alo, t, h);
            proxy_fence();
            tc_fence_before();
            __syncthreads();
        } else if (row < n) {
#pragma unroll
            for (int o = 0; o < OUT; ++o) {
                float z = S.bias[3 * H + o];
#pragma unroll
                for (int k = 0; k < H; ++k) z = fmaf(h[k], S.w4[o][k], z);
                Y[row * OUT + o] = z;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
    }
}

// ---------------------------------------------------------------------------
// tensor-core training: the loss of a minibatch and its gradient
// ---------------------------------------------------------------------------
// One CTA of 128 threads holds 128 samples, one per thread (the rows of every
// forward and propagation MMA, M = 128).  Forward as the inference kernel
// (hi + lo activations, FP32 last layer).  Backward:
//   * the last layer's gradient in FP32 on the CUDA cores;
//   * dz_(l-1) = (dz_l W_l) * SiLU'(z_(l-1)) on the tensor cores: A = dz_l as
//     hi + lo terms, B = W_l transposed (exact BF16), with z_(l-1) recomputed by
//     the layer's forward MMA from the stored input tile;
//   * dW_l = dz_l^T a_(l-1) and the bias gradient on the tensor cores with the
//     samples as K: A = dz_l^T (hi + lo; rows 64..127 zero, so M = 128),
//     B = a_(l-1)^T in BF16 plus a row of ones (its column of D is the bias
//     gradient); each CTA adds its partial gradient into the global one.
// The weights are the BF16 roundings of the FP32 parameters, as in the FP32
// training kernel (straight-through).
constexpr int kTrK = 128;   // samples per CTA: K of the weight-gradient MMAs
constexpr int kTrNW = 80;   // N of the weight-gradient MMAs: 64 inputs, a row of ones, zero rows
constexpr int kTrN1 = 16;   // the same for layer 1: 8 inputs, a row of ones, zero rows
constexpr int kTrCols = 128;  // TMEM columns allocated

struct TrainTcShared {
    unsigned char w1f[H * 16 * 2];                  // forward B of layer 1: [j][k], k 8..15 repeat 0..7
    unsigned char w2f[H * H * 2], w3f[H * H * 2];   // forward B: [j][k]
    unsigned char w2b[H * H * 2], w3b[H * H * 2];   // propagation B: [k][j] (transposed)
    unsigned char x[kTcRows * 16 * 2];              // layer-1 A: features hi | lo
    unsigned char a1[kTcRows * H * 2], a1lo[kTcRows * H * 2];
    unsigned char a2[kTcRows * H * 2], a2lo[kTcRows * H * 2];
    unsigned char dz[kTcRows * H * 2], dzlo[kTcRows * H * 2];      // propagation A: [s][j]; first a3 (FP32)
    unsigned char dzt[kTcRows * kTrK * 2], dztlo[kTcRows * kTrK * 2];  // weight-gradient A: [j][s]
    unsigned char act[kTrNW * kTrK * 2];            // weight-gradient B: [k][s]
    float b[3 * H + OUT];
    float w4[OUT][H];
    float g4[kTcRows][OUT];
    float red[kTcRows / 32];
    uint64_t bar;
    uint32_t tmem;
    int timeout;
};
static_assert(sizeof(float) * kTcRows * H <= 2 * kTcRows * H * 2, "a3 fits the propagation A tiles");

__device__ __forceinline__ void put_bf16(unsigned char *tile, int r, int k, int K, float v)
{
    *reinterpret_cast<__nv_bfloat16 *>(tile + core_offset(r, k, K)) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float silu_d(float z)
{
    const float sg = 1.f / (1.f + expf(-z));
    return sg * (1.f + z * (1.f - sg));
}

// this thread's row of 64 FP32 values back from its hi and lo tiles
__device__ __forceinline__ void get_row64(const unsigned char *a, const unsigned char *alo, int r, float *h)
{
#pragma unroll
    for (int k = 0; k < H; ++k)
        h[k] = __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(a + core_offset(r, k, H))) +
               __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(alo + core_offset(r, k, H)));
}

__global__ void __launch_bounds__(kTcRows) k_mlp_grad_tc(const float *__restrict__ P, const float *__restrict__ X,
                                                         const float *__restrict__ Yt, int64_t n,
                                                         float *__restrict__ G, float *__restrict__ loss,
                                                         uint32_t *status)
{
    extern __shared__ __align__(1024) unsigned char smem_tr[];
    TrainTcShared &S = *reinterpret_cast<TrainTcShared *>(smem_tr + ((1024u - (smem_addr(smem_tr) & 1023u)) & 1023u));
    const int t = threadIdx.x, warp = t >> 5;
    const int64_t row = (int64_t)blockIdx.x * kTcRows + t;
    const bool valid = row < n;
    // weights as BF16 operand tiles (forward and transposed), biases and W4 in FP32
    for (int q = t; q < H * 16; q += kTcRows) put_bf16(S.w1f, q / 16, q % 16, 16, P[oW1 + (q / 16) * IN + (q % 16) % IN]);
    for (int q = t; q < H * H; q += kTcRows) {
        const int j = q / H, k = q % H;
        put_bf16(S.w2f, j, k, H, P[oW2 + q]);
        put_bf16(S.w3f, j, k, H, P[oW3 + q]);
        put_bf16(S.w2b, k, j, H, P[oW2 + q]);
        put_bf16(S.w3b, k, j, H, P[oW3 + q]);
    }
    for (int q = t; q < H; q += kTcRows) {
        S.b[q] = P[oB1 + q];
        S.b[H + q] = P[oB2 + q];
        S.b[2 * H + q] = P[oB3 + q];
    }
    if (t < OUT) S.b[3 * H + t] = P[oB4 + t];
    for (int q = t; q < OUT * H; q += kTcRows) S.w4[q / H][q % H] = P[oW4 + q];
    // the weight-gradient tiles start at zero (their padding rows stay zero)
    {
        uint4 *z0 = reinterpret_cast<uint4 *>(S.dzt), *z1 = reinterpret_cast<uint4 *>(S.dztlo);
        uint4 *z2 = reinterpret_cast<uint4 *>(S.act);
        const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
        for (int q = t; q < (int)(sizeof(S.dzt) / 16); q += kTcRows) { z0[q] = zero; z1[q] = zero; }
        for (int q = t; q < (int)(sizeof(S.act) / 16); q += kTcRows) z2[q] = zero;
    }
    // this row's features (hi | lo) and targets
    float f[IN], yt[OUT];
#pragma unroll
    for (int k = 0; k < IN; ++k) f[k] = valid ? X[row * IN + k] : 0.f;
#pragma unroll
    for (int o = 0; o < OUT; ++o) yt[o] = valid ? Yt[row * OUT + o] : 0.f;
    {
        __nv_bfloat162 v[4], w[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) split_bf16(f[2 * c], f[2 * c + 1], v[c], w[c]);
        *reinterpret_cast<uint4 *>(S.x + core_offset(t, 0, 16)) = *reinterpret_cast<uint4 *>(v);
        *reinterpret_cast<uint4 *>(S.x + core_offset(t, 8, 16)) = *reinterpret_cast<uint4 *>(w);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&S.tmem)),
                     "r"(kTrCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) { mbar_init(&S.bar, 1); S.timeout = 0; }
    unsigned phase = 0;
    uint32_t tmem = 0;
    // one MMA group: every thread's operand writes published, one elected thread
    // issues the K loop over the A terms, every thread waits for the commit
    auto gemm = [&](const unsigned char *a0, const unsigned char *a1p, const unsigned char *b, int K, int N) {
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        tmem = S.tmem;
        if (t == 0 && !S.timeout) {
            tc_fence_after();
            const uint32_t id = idesc_bf16(N);
            const unsigned char *as[2] = {a0, a1p};
            int acc = 0;
            for (int term = 0; term < (a1p ? 2 : 1); ++term)
                for (int kk = 0; kk < K / 16; ++kk) {
                    const uint64_t ad = smem_desc(as[term] + kk * 256, 128, (K / 8) * 128);
                    const uint64_t bd = smem_desc(b + kk * 256, 128, (K / 8) * 128);
                    tc_mma(tmem, ad, bd, id, acc);
                    acc = 1;
                }
            tc_commit(&S.bar);
        }
        if (!mbar_wait_bounded(&S.bar, phase)) {
            S.timeout = 1;
            raise_status(status, MPMW_ST_TIMEOUT);
        }
        phase ^= 1u;
        tc_fence_after();
    };
    // this thread's row (a sample) of an M = 128 result: N columns
    auto ld_row = [&](float *v, int N) {
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
        for (int c = 0; c < N; c += 16) tc_ld16(lane_addr + (uint32_t)c, v + c);
        tc_wait_ld();
    };
    // the weight-gradient result: rows j = 0..63 (warps 0 and 1), N columns;
    // columns < nin are dW[j][c], column nin the bias gradient
    auto add_dw = [&](int oW, int oB, int nin, int N) {
        if (warp < 2) {
            const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
            const int j = t;
            for (int c0 = 0; c0 < N; c0 += 16) {
                float v[16];
                tc_ld16(lane_addr + (uint32_t)c0, v);
                tc_wait_ld();
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int col = c0 + c;
                    if (col < nin) atomicAdd(&G[oW + j * nin + col], v[c]);
                    else if (col == nin) atomicAdd(&G[oB + j], v[c]);
                }
            }
        }
    };
    float h[H], d[H];
    // ---- forward ----
    gemm(S.x, nullptr, S.w1f, 16, H);
    ld_row(h, H);
#pragma unroll
    for (int j = 0; j < H; ++j) { const float z = h[j] + S.b[j]; h[j] = z / (1.f + expf(-z)); }
    put_row64(S.a1, S.a1lo, t, h);
    gemm(S.a1, S.a1lo, S.w2f, H, H);
    ld_row(h, H);
#pragma unroll
    for (int j = 0; j < H; ++j) { const float z = h[j] + S.b[H + j]; h[j] = z / (1.f + expf(-z)); }
    put_row64(S.a2, S.a2lo, t, h);
    gemm(S.a2, S.a2lo, S.w3f, H, H);
    ld_row(h, H);
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const float z = h[j] + S.b[2 * H + j];
        d[j] = silu_d(z);
        h[j] = z / (1.f + expf(-z));   // a3
    }
    // ---- loss, last layer (FP32) ----
    const float inv = 2.f / (float)((double)n * OUT);
    float lsum = 0.f, g4[OUT];
#pragma unroll
    for (int o = 0; o < OUT; ++o) {
        float z = S.b[3 * H + o];
#pragma unroll
        for (int k = 0; k < H; ++k) z = fmaf(h[k], S.w4[o][k], z);
        const float r = valid ? z - yt[o] : 0.f;
        lsum = fmaf(r, r, lsum);
        g4[o] = inv * r;
        S.g4[t][o] = g4[o];
    }
    float(*a3s)[H] = reinterpret_cast<float(*)[H]>(S.dz);
#pragma unroll
    for (int k = 0; k < H; ++k) a3s[t][k] = h[k];
    // dz3 = (g4 W4) * SiLU'(z3)
#pragma unroll
    for (int j = 0; j < H; ++j) {
        float g = 0.f;
#pragma unroll
        for (int o = 0; o < OUT; ++o) g = fmaf(g4[o], S.w4[o][j], g);
        d[j] *= g;
    }
    __syncthreads();
    for (int q = t; q < OUT * H; q += kTcRows) {
        const int o = q / H, k = q % H;
        float acc = 0.f;
        for (int r = 0; r < kTcRows; ++r) acc = fmaf(S.g4[r][o], a3s[r][k], acc);
        atomicAdd(&G[oW4 + q], acc);
    }
    if (t < OUT) {
        float acc = 0.f;
        for (int r = 0; r < kTcRows; ++r) acc += S.g4[r][t];
        atomicAdd(&G[oB4 + t], acc);
    }
    // loss
    {
        float v = lsum;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((t & 31) == 0) S.red[warp] = v;
    }
    __syncthreads();   // a3s and g4 read, the loss partials written
    if (t == 0) {
        float v = 0.f;
        for (int w = 0; w < kTcRows / 32; ++w) v += S.red[w];
        atomicAdd(loss, v / (float)((double)n * OUT));
    }
    // the weight-gradient operands of one layer: dz^T (hi, lo) in column t,
    // the layer's input (BF16) in column t, the ones row
    auto put_dw_operands = [&](const float *dzv, const float *in, int nin) {
#pragma unroll
        for (int j = 0; j < H; ++j) {
            const __nv_bfloat16 hi = __float2bfloat16_rn(dzv[j]);
            *reinterpret_cast<__nv_bfloat16 *>(S.dzt + core_offset(j, t, kTrK)) = hi;
            *reinterpret_cast<__nv_bfloat16 *>(S.dztlo + core_offset(j, t, kTrK)) =
                __float2bfloat16_rn(dzv[j] - __bfloat162float(hi));
        }
        for (int k = 0; k < nin; ++k) put_bf16(S.act, k, t, kTrK, in[k]);
        put_bf16(S.act, nin, t, kTrK, 1.f);
    };
    // ---- layer 3: dW3, db3; dz2 ----
    get_row64(S.a2, S.a2lo, t, h);            // a2
    put_dw_operands(d, h, H);
    gemm(S.dzt, S.dztlo, S.act, kTrK, kTrNW);
    add_dw(oW3, oB3, H, kTrNW);
    put_row64(S.dz, S.dzlo, t, d);            // dz3 as propagation A
    gemm(S.a1, S.a1lo, S.w2f, H, H);          // z2 again
    ld_row(h, H);
#pragma unroll
    for (int k = 0; k < H; ++k) h[k] = silu_d(h[k] + S.b[H + k]);
    gemm(S.dz, S.dzlo, S.w3b, H, H);          // dz3 W3
    ld_row(d, H);
#pragma unroll
    for (int k = 0; k < H; ++k) d[k] *= h[k];  // dz2
    // ---- layer 2: dW2, db2; dz1 ----
    get_row64(S.a1, S.a1lo, t, h);            // a1
    put_dw_operands(d, h, H);
    gemm(S.dzt, S.dztlo, S.act, kTrK, kTrNW);
    add_dw(oW2, oB2, H, kTrNW);
    put_row64(S.dz, S.dzlo, t, d);            // dz2 as propagation A
    gemm(S.x, nullptr, S.w1f, 16, H);         // z1 again
    ld_row(h, H);
#pragma unroll
    for (int k = 0; k < H; ++k) h[k] = silu_d(h[k] + S.b[k]);
    gemm(S.dz, S.dzlo, S.w2b, H, H);          // dz2 W2
    ld_row(d, H);
#pragma unroll
    for (int k = 0; k < H; ++k) d[k] *= h[k];  // dz1
    // ---- layer 1: dW1, db1 (inputs: the features, then ones, then zeros) ----
    {
        float in[kTrN1];
#pragma unroll
        for (int k = 0; k < kTrN1; ++k) in[k] = k < IN ? f[k] : 0.f;
        put_dw_operands(d, in, kTrN1 - 1);     // rows 8..14 zero, row 15 ones
    }
    gemm(S.dzt, S.dztlo, S.act, kTrK, kTrN1);
    if (warp < 2) {
        float v[kTrN1];
        const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
        tc_ld16(lane_addr, v);
        tc_wait_ld();
#pragma unroll
        for (int c = 0; c < IN; ++c) atomicAdd(&G[oW1 + t * IN + c], v[c]);
        atomicAdd(&G[oB1 + t], v[kTrN1 - 1]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTrCols) : "memory");
    }
}

}  // namespace mlp
}  // namespace mpmw

using namespace mpmw;
using namespace mpmw::mlp;

static bool g_mlp_attr[64];

static int set_smem_attrs()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { set_error("mlp: no current device"); return MPMW_E_DEVICE; }
    if (dev >= 0 && dev < 64 && !g_mlp_attr[dev]) {
        const int ts = (int)sizeof(TrainShared), tc = (int)sizeof(TcShared) + 1024;
        const int tr = (int)sizeof(TrainTcShared) + 1024;
        if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, ts) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, ts) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tr) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc) != cudaSuccess) {
            set_error("mlp: cannot reserve shared memory");
            return MPMW_E_DEVICE;
        }
        g_mlp_attr[dev] = true;
    }
    return MPMW_OK;
}

extern "C" {

int mpmw_dp_samples(int64_t n, uint64_t seed, float *x, float *y, mpmw_stream_t stream)
{
    if (n < 0 || (n > 0 && (!x || !y))) { set_error("dp_samples: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "dp_samples")) return MPMW_E_ARG;
    if (n == 0) return MPMW_OK;
    k_dp_samples<<<grid_for(n), kBlock, 0, as_stream(stream)>>>(n, seed, x, y);
    return check_launch("k_dp_samples");
}

int mpmw_mlp_forward(const float *params, const float *x, int64_t n, float *y, mpmw_stream_t stream)
{
    if (!params || n < 0 || (n > 0 && (!x || !y))) { set_error("mlp_forward: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "mlp_forward")) return MPMW_E_ARG;
    if (n == 0) return MPMW_OK;
    { int rc_ = set_smem_attrs(); if (rc_ != MPMW_OK) return rc_; }
    const unsigned g = (unsigned)((n + kTile - 1) / kTile);
    k_mlp_forward<<<g, kThreads, sizeof(TrainShared), as_stream(stream)>>>(params, x, n, y);
    return check_launch("k_mlp_forward");
}

int mpmw_mlp_grad(const float *params, const float *x, const float *y, int64_t n, float *grad, float *loss,
                  mpmw_stream_t stream)
{
    if (!params || !grad || !loss || n <= 0 || !x || !y) { set_error("mlp_grad: bad arguments"); return MPMW_E_ARG; }
    { int rc_ = set_smem_attrs(); if (rc_ != MPMW_OK) return rc_; }
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(grad, 0, NP * sizeof(float), s) != cudaSuccess ||
        cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) {
        set_error("mlp_grad: memset failed");
        return MPMW_E_DEVICE;
    }
    const unsigned g = (unsigned)((n + kTile - 1) / kTile);
    k_mlp_grad<<<g, kThreads, sizeof(TrainShared), s>>>(params, x, y, n, grad, loss);
    return check_launch("k_mlp_grad");
}

int mpmw_mlp_grad_tc(const float *params, const float *x, const float *y, int64_t n, float *grad, float *loss,
                     uint32_t *status, mpmw_stream_t stream)
{
    if (!params || !grad || !loss || n <= 0 || !x || !y) { set_error("mlp_grad_tc: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "mlp_grad_tc")) return MPMW_E_ARG;
    { int rc_ = set_smem_attrs(); if (rc_ != MPMW_OK) return rc_; }
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(grad, 0, NP * sizeof(float), s) != cudaSuccess ||
        cudaMemsetAsync(loss, 0, sizeof(float), s) != cudaSuccess) {
        set_error("mlp_grad_tc: memset failed");
        return MPMW_E_DEVICE;
    }
    const unsigned g = (unsigned)((n + kTcRows - 1) / kTcRows);
    k_mlp_grad_tc<<<g, kTcRows, sizeof(TrainTcShared) + 1024, s>>>(params, x, y, n, grad, loss, status);
    return check_launch("k_mlp_grad_tc");
}

int mpmw_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, mpmw_stream_t stream)
{
    if (!params || !grad || !m || !v || step < 1) { set_error("mlp_adam: bad arguments"); return MPMW_E_ARG; }
    const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
    k_mlp_adam<<<(NP + 255) / 256, 256, 0, as_stream(stream)>>>(params, grad, m, v, lr, c1, c2);
    return check_launch("k_mlp_adam");
}

int mpmw_mlp_pack(const float *params, void *packed, mpmw_stream_t stream)
{
    if (!params || !packed) { set_error("mlp_pack: bad arguments"); return MPMW_E_ARG; }
    if ((reinterpret_cast<uintptr_t>(packed) & 15u) != 0) { set_error("mlp_pack: packed must be 16-byte aligned"); return MPMW_E_ARG; }
    cudaStream_t s = as_stream(stream);
    if (cudaMemsetAsync(packed, 0, MPMW_MLP_PACKED_BYTES, s) != cudaSuccess) { set_error("mlp_pack: memset failed"); return MPMW_E_DEVICE; }
    k_mlp_pack<<<(H * H + 255) / 256, 256, 0, s>>>(params, reinterpret_cast<__nv_bfloat16 *>(packed));
    return check_launch("k_mlp_pack");
}

int mpmw_mlp_infer_tc(const void *packed, const float *params, const float *x, int64_t n, float *y,
                      uint32_t *status, mpmw_stream_t stream)
{
    if (!packed || !params || n < 0 || (n > 0 && (!x || !y))) { set_error("mlp_infer_tc: bad arguments"); return MPMW_E_ARG; }
    if (count_too_large(n, "mlp_infer_tc")) return MPMW_E_ARG;
    if ((reinterpret_cast<uintptr_t>(packed) & 15u) != 0) { set_error("mlp_infer_tc: packed must be 16-byte aligned"); return MPMW_E_ARG; }
    if (n == 0) return MPMW_OK;
    { int rc_ = set_smem_attrs(); if (rc_ != MPMW_OK) return rc_; }
    const unsigned g = (unsigned)((n + kTcRows - 1) / kTcRows);
    k_mlp_infer_tc<<<g, kTcRows, sizeof(TcShared) + 1024, as_stream(stream)>>>(
        static_cast<const unsigned char *>(packed), params, x, n, y, status, nullptr);
    return check_launch("k_mlp_infer_tc");
}

}  // extern "C"

namespace mpmw {
// the inference kernel over a worklist whose length is on the device
int launch_mlp_infer_tc_dev(const void *packed, const float *params, const float *x, int64_t n_max, const int *n_dev,
                            float *y, uint32_t *status, cudaStream_t s)
{
    if (n_max <= 0) return MPMW_OK;
    { int rc_ = set_smem_attrs(); if (rc_ != MPMW_OK) return rc_; }
    const unsigned g = (unsigned)((n_max + mlp::kTcRows - 1) / mlp::kTcRows);
    mlp::k_mlp_infer_tc<<<g, mlp::kTcRows, sizeof(mlp::TcShared) + 1024, s>>>(
        static_cast<const unsigned char *>(packed), params, x, n_max, y, status, n_dev);
    return check_launch("k_mlp_infer_tc");
}
}  // namespace mpmw

extern "C" {

}  // extern "C"
