// mpmw_scatter.cuh -- CTA-cooperative APIC particle-to-grid scatter (reference:
// utils/mpmRoutines.py:485-569 p2g_apic_with_stress), shared by the P2G kernel
// and the fused G2P->P2G kernel.
//
// For the kScatterChunk particles of a CTA (one per thread; `act` marks those
// that scatter):
//   1. scattering particles are counting-sorted by stencil base cell (the
//      reference's truncated base index, bit-exact) over the CTA's bounding box
//      of base cells; all particles of one base cell form one segment -- they
//      scatter to the same 27 nodes -- whatever their order in memory, so
//      particles that drift across cell boundaries between global sorts do not
//      fragment the segments.  A CTA whose box has more than kScatterBins cells
//      compacts instead, and runs of equal base in memory order form segments;
//   2. each particle stores its B-spline weights and per-particle constants in
//      shared memory at its sorted slot: 8 float4 (swizzled so that particles
//      about 8 apart fall in different banks) laid out as the packed FP32 FMA
//      wants its operand pairs (z weights duplicated, stress and momentum
//      components side by side), and its x and y weights as (w, dw) pairs that
//      a column (i, j) indexes directly;
//   3. one thread per (segment, i, j) stencil column sums its particles'
//      contributions to the column's 3 nodes in registers, for as many complete
//      passes over the threads as there are; each column left over is shared by
//      a group of lanes of one warp, which combine their partial sums with
//      shuffles before one of them adds the column;
//   4. each column adds its 3 nodes into the grid with one float4 global
//      atomic per node.  The accumulator grid stays resident in L2, and adding
//      a column there costs 3 vector atomics where a shared-memory tile costs
//      12 scalar float atomics plus a zeroing pass and a flush; on the B200 the
//      tile variant was measured about 11 % slower for the whole fused substep.
//      Any particle order is correct; particles sorted by base cell make
//      segments long and so the atomics few.
//
// Contribution of particle p to node (i,j,k) (quadratic B-spline, fx = grid
// position - base):
//   m:   w_ijk m
//   m v: w_ijk (a + i Bx + j By + k Bz) + S (dwx_i wy_j wz_k, wx_i dwy_j wz_k, wx_i wy_j dwz_k)
// with B = m C' dx (columns Bx, By, Bz), a = m v - B fx, S = -dt vol inv_dx stress,
// C' = (1 - r) C + (r/2)(C - C^T) (C' = 0 when r < -0.001).
#pragma once
#include "mpmw_common.cuh"
#include "mpmw_math.cuh"
#include "mpmw_scan.cuh"

namespace mpmw {

// Particles (and threads) per CTA of the scattering kernels.  128 rather than
// 256: the same 24 warps per SM (6 CTAs at 80 registers), but each CTA barrier
// waits for 4 warps instead of 8; measured 3.7 % faster for the fused substep
// on the tunnel.  The shared memory of 6 CTAs must fit an SM: hence 512
// counting-sort bins (a 128-particle CTA spans far fewer base cells).
constexpr int kScatterChunk = 128;
constexpr int kScatterCtasPerSm = 768 / kScatterChunk;  // resident CTAs the launch bounds aim at (80 registers)
constexpr int kScatterBins = 512;    // base cells of a CTA's box that the counting sort handles

constexpr int kScatterRec = 8;       // float4 records per particle

struct ScatterShared {
    float4 rec[kScatterRec][kScatterChunk];  // per compacted particle (swizzled slot)
    // x and y weights of slot q: (wx_i, dwx_i) at 7q + i, (wy_j, dwy_j) at
    // 7q + 3 + j.  The odd stride puts the lanes that read one particle for
    // different columns in different banks.
    float2 wxy[kScatterChunk * 7];
    int base[3][kScatterChunk];
    int seg_start[kScatterChunk + 1];
    int wsum[kScatterChunk / 32];    // warp totals of the counting sort's scan
    int outside;                     // a particle's base fell outside a known box
    int bins[kScatterBins];          // counting-sort bins over the box of base cells
    int lo[3], hi[3];
};

__device__ __forceinline__ int scatter_slot(int k) { return k ^ ((k >> 3) & 7); }

// Register sums of one stencil column (i, j) of one segment: the 3 nodes
// k = 0..2 of (m, m vx, m vy, m vz).  The x and y momentum components (and
// the masses of nodes 0 and 1) are summed as float2 pairs with the packed FP32
// FMA; every component sees the same operations and roundings as the scalar
// form fma(w_k, P_k, fma(dw_k, R, acc)).
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

struct ColumnSums {
    float2 m01, axy[3];
    float m2, az[3];

    __device__ __forceinline__ void zero()
    {
        m01 = make_float2(0.f, 0.f);
        m2 = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) { axy[k] = make_float2(0.f, 0.f); az[k] = 0.f; }
    }

    // add the contribution of the particle in record slot q to column ij.
    // Record (see put_record): rec[0] = (wz0 wz0 wz1 wz1), rec[1] = (wz2 wz2
    // dwz0 dwz0), rec[2] = (dwz1 dwz1 dwz2 dwz2), rec[3] = (s00 s01 s01 s11),
    // rec[4] = (s02 s12 s22 m), rec[5] = (a0 a1 Bx0 Bx1), rec[6] = (By0 By1
    // Bz0 Bz1), rec[7] = (a2 Bx2 By2 Bz2).
    template <class Shared>
    __device__ __forceinline__ void add(const Shared &S, int q, int i, int j, float2 fi2, float2 fj2)
    {
        const float2 xw = S.wxy[7 * q + i], yw = S.wxy[7 * q + 3 + j];
        const float wxi = xw.x, dwxi = xw.y, wyj = yw.x, dwyj = yw.y;
        const float4 z0 = S.rec[0][q], z1 = S.rec[1][q], z2 = S.rec[2][q], sa = S.rec[3][q], sb = S.rec[4][q],
                     u0 = S.rec[5][q], u1 = S.rec[6][q], u2 = S.rec[7][q];
        const float wxy = wxi * wyj, g0 = dwxi * wyj, g1 = wxi * dwyj, wm = wxy * sb.w;
        const float2 wxy2 = dup2(wxy);
        // A = a + i Bx + j By
        const float2 A01 = __ffma2_rn(fj2, make_float2(u1.x, u1.y),
                                      __ffma2_rn(fi2, make_float2(u0.z, u0.w), make_float2(u0.x, u0.y)));
        const float A2 = fma_(fj2.x, u2.z, fma_(fi2.x, u2.y, u2.x));
        // Q = S (g0, g1, 0), R = wxy S[:,2]
        const float2 Q01 = __ffma2_rn(make_float2(sa.x, sa.y), dup2(g0), __fmul2_rn(make_float2(sa.z, sa.w), dup2(g1)));
        const float Q2 = fma_(sb.x, g0, sb.y * g1);
        const float2 R01 = __fmul2_rn(wxy2, make_float2(sb.x, sb.y));
        const float R2 = wxy * sb.z;
        // P_k = wxy (A + k Bz) + Q
        float2 P01 = __ffma2_rn(wxy2, A01, Q01);
        float P2 = fma_(wxy, A2, Q2);
        const float2 dz01 = __fmul2_rn(wxy2, make_float2(u1.z, u1.w));
        const float dz2 = wxy * u2.w;
        m01.x = fma_(z0.x, wm, m01.x);
        m01.y = fma_(z0.z, wm, m01.y);
        m2 = fma_(z1.x, wm, m2);
        const float2 wz[3] = {make_float2(z0.x, z0.y), make_float2(z0.z, z0.w), make_float2(z1.x, z1.y)};
        const float2 dwz[3] = {make_float2(z1.z, z1.w), make_float2(z2.x, z2.y), make_float2(z2.z, z2.w)};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (k > 0) { P01 = __fadd2_rn(P01, dz01); P2 = P2 + dz2; }
            axy[k] = __ffma2_rn(wz[k], P01, __ffma2_rn(dwz[k], R01, axy[k]));
            az[k] = fma_(wz[k].x, P2, fma_(dwz[k].x, R2, az[k]));
        }
    }

    // add the sums of lane (this lane ^ o) of the warp (every lane must call)
    __device__ __forceinline__ void shfl_add(int o)
    {
        constexpr unsigned kAll = 0xffffffffu;
        m01.x += __shfl_xor_sync(kAll, m01.x, o);
        m01.y += __shfl_xor_sync(kAll, m01.y, o);
        m2 += __shfl_xor_sync(kAll, m2, o);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            axy[k].x += __shfl_xor_sync(kAll, axy[k].x, o);
            axy[k].y += __shfl_xor_sync(kAll, axy[k].y, o);
            az[k] += __shfl_xor_sync(kAll, az[k], o);
        }
    }

    // add the column's 3 nodes into the grid
    template <class Shared>
    __device__ __forceinline__ void emit(const Shared &S, int k0, int ij, float4 *__restrict__ gmv, int nx, int ny,
                                         int nz, uint32_t &bad) const
    {
        const int i = ij / 3, j = ij - 3 * (ij / 3);
        const int gx = S.base[0][k0] + i, gy = S.base[1][k0] + j, gz0 = S.base[2][k0];
        const float mk[3] = {m01.x, m01.y, m2};
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
            const int gz = gz0 + kk;
            if (gx < 0 || gy < 0 || gz < 0 || gx >= nx || gy >= ny || gz >= nz) { bad |= MPMW_ST_OOB; continue; }
            atomicAdd(&gmv[((int64_t)gx * ny + gy) * nz + gz], make_float4(mk[kk], axy[kk].x, axy[kk].y, az[kk]));
        }
    }
};

// A box of base cells that the caller knows to hold the base of every
// scattering particle (lo and extents, at most kScatterBins cells), so the
// scatter need not reduce one.  The caller zeroes S.bins and S.outside before
// a barrier every thread passes before this call.  A particle found outside
// the box sets S.outside, and the CTA then forms its segments by compaction.
struct ScatterBox {
    int lo[3], ext[3];
};

// Every thread of the CTA must call this (it synchronizes the block), once per
// CTA: the box bounds S.lo/S.hi are reset before the first barrier.
// xp: position; v: velocity; C: velocity gradient (row-major); st6: symmetric
// stress xx yy zz xy xz yz; m, vol: mass and volume.  Values of threads with
// act == false are ignored.  Out-of-grid nodes are skipped and flagged in `bad`.
__device__ __forceinline__ void p2g_scatter(ScatterShared &S, bool act, const float *xp, const float *v,
                                            const float *C0, const float *st6, float m, float vol,
                                            const mpmw_params_t &prm, float4 *__restrict__ gmv, int nx, int ny,
                                            int nz, uint32_t &bad, const ScatterBox *known = nullptr)
{
    const int t = threadIdx.x;
    int *bins = S.bins;
    // stencil base cell, as weights() computes it
    int b0 = 0, b1 = 0, b2 = 0;
    if (act) {
        b0 = (int)((xp[0] - prm.min_bounds[0]) * prm.inv_dx - 0.5f);
        b1 = (int)((xp[1] - prm.min_bounds[1]) * prm.inv_dx - 0.5f);
        b2 = (int)((xp[2] - prm.min_bounds[2]) * prm.inv_dx - 0.5f);
    }
    // the box of base cells the counting sort runs over, and each particle's
    // bin and rank in it
    int o0, o1, o2;
    int64_t bey, bez, nb;
    int key = 0, rank = 0;
    bool use_bins;
    if (known) {
        o0 = known->lo[0]; o1 = known->lo[1]; o2 = known->lo[2];
        bey = known->ext[1]; bez = known->ext[2];
        nb = (int64_t)known->ext[0] * bey * bez;
        if (act) {
            const int64_t r0 = (int64_t)b0 - o0, r1 = (int64_t)b1 - o1, r2 = (int64_t)b2 - o2;
            if (r0 >= 0 && r1 >= 0 && r2 >= 0 && r0 < known->ext[0] && r1 < bey && r2 < bez) {
                key = (int)((r0 * bey + r1) * bez + r2);
                rank = atomicAdd(&bins[key], 1);
            } else {
                S.outside = 1;
            }
        }
        __syncthreads();  // bins counted, outside flag set
        use_bins = S.outside == 0;
    } else {
        if (t < 3) { S.lo[t] = INT32_MAX; S.hi[t] = INT32_MIN; }  // nothing before this call uses them
        __syncthreads();  // the rest of S may still be in use by the caller's previous phase
        for (int q = t; q < kScatterBins; q += kScatterChunk) bins[q] = 0;
        {
            int lo0 = act ? b0 : INT32_MAX, lo1 = act ? b1 : INT32_MAX, lo2 = act ? b2 : INT32_MAX;
            int hi0 = act ? b0 : INT32_MIN, hi1 = act ? b1 : INT32_MIN, hi2 = act ? b2 : INT32_MIN;
            lo0 = __reduce_min_sync(0xffffffffu, lo0); lo1 = __reduce_min_sync(0xffffffffu, lo1); lo2 = __reduce_min_sync(0xffffffffu, lo2);
            hi0 = __reduce_max_sync(0xffffffffu, hi0); hi1 = __reduce_max_sync(0xffffffffu, hi1); hi2 = __reduce_max_sync(0xffffffffu, hi2);
            if ((t & 31) == 0) {
                atomicMin(&S.lo[0], lo0); atomicMin(&S.lo[1], lo1); atomicMin(&S.lo[2], lo2);
                atomicMax(&S.hi[0], hi0); atomicMax(&S.hi[1], hi1); atomicMax(&S.hi[2], hi2);
            }
        }
        __syncthreads();
        if (S.lo[0] == INT32_MAX) return;  // nothing scatters (uniform)
        o0 = S.lo[0]; o1 = S.lo[1]; o2 = S.lo[2];
        bey = (int64_t)S.hi[1] - o1 + 1;
        bez = (int64_t)S.hi[2] - o2 + 1;
        nb = ((int64_t)S.hi[0] - o0 + 1) * bey * bez;
        use_bins = nb <= kScatterBins;
        if (use_bins) {
            key = act ? (int)(((b0 - o0) * bey + (b1 - o1)) * bez + (b2 - o2)) : 0;
            rank = act ? atomicAdd(&bins[key], 1) : 0;
            __syncthreads();
        }
    }
    int nact, nseg;
    {
        // record of this particle, written at `slot`
        auto put_record = [&](int slot) {
            Weights W;
            weights(xp, prm.min_bounds, prm.inv_dx, W);
            const float r = prm.rpic_damping;
            float Cp[9];
            if (r == 0.f) {
                // (1 - 0) C + 0 (C - C^T) = C for finite C (up to the sign of an
                // exact zero): a uniform shortcut for the undamped default
#pragma unroll
                for (int q = 0; q < 9; ++q) Cp[q] = C0[q];
            } else {
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb)
                        Cp[3 * aa + bb] = (1.f - r) * C0[3 * aa + bb] + (r / 2.f) * (C0[3 * aa + bb] - C0[3 * bb + aa]);
            }
            if (r < -0.001f) {
#pragma unroll
                for (int q = 0; q < 9; ++q) Cp[q] = 0.f;
            }
            const float mdx = m * prm.dx;
            float B[9];  // B[3*row + col] = m C'[row][col] dx
#pragma unroll
            for (int q = 0; q < 9; ++q) B[q] = Cp[q] * mdx;
            float av[3];
#pragma unroll
            for (int row = 0; row < 3; ++row)
                av[row] = fma_(-B[3 * row + 0], W.fx[0], fma_(-B[3 * row + 1], W.fx[1], fma_(-B[3 * row + 2], W.fx[2], m * v[row])));
            const float sc = -(prm.dt * vol) * prm.inv_dx;
            const int q = scatter_slot(slot);
            const float s00 = sc * st6[0], s11 = sc * st6[1], s22 = sc * st6[2], s01 = sc * st6[3],
                        s02 = sc * st6[4], s12 = sc * st6[5];
            // Bx = column 0 of B (B[0], B[3], B[6]), By = column 1, Bz = column 2
            S.rec[0][q] = make_float4(W.w[2][0], W.w[2][0], W.w[2][1], W.w[2][1]);
            S.rec[1][q] = make_float4(W.w[2][2], W.w[2][2], W.dw[2][0], W.dw[2][0]);
            S.rec[2][q] = make_float4(W.dw[2][1], W.dw[2][1], W.dw[2][2], W.dw[2][2]);
            S.rec[3][q] = make_float4(s00, s01, s01, s11);
            S.rec[4][q] = make_float4(s02, s12, s22, m);
            S.rec[5][q] = make_float4(av[0], av[1], B[0], B[3]);
            S.rec[6][q] = make_float4(B[1], B[4], B[2], B[5]);
            S.rec[7][q] = make_float4(av[2], B[6], B[7], B[8]);
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                S.wxy[7 * q + e] = make_float2(W.w[0][e], W.dw[0][e]);
                S.wxy[7 * q + 3 + e] = make_float2(W.w[1][e], W.dw[1][e]);
            }
            S.base[0][slot] = W.base[0]; S.base[1][slot] = W.base[1]; S.base[2][slot] = W.base[2];
        };
        if (use_bins) {
            // counting sort of the scattering particles by base cell: all the
            // CTA's particles of one base cell form one segment, whatever their
            // order in memory (particles drift across cell boundaries)
            constexpr int kPer = kScatterBins / kScatterChunk;
            int c[kPer], pc = 0, ne = 0;
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int idx = kPer * t + u;
                c[u] = idx < nb ? bins[idx] : 0;
                pc += c[u];
                ne += c[u] > 0 ? 1 : 0;
            }
            // one scan of (nonempty bins << 16 | particles): both prefix sums at once
            int tot;
            const int ex0 = block_excl_scan_1bar<kScatterChunk>((ne << 16) | pc, &tot, S.wsum);
            nact = tot & 0xFFFF;
            nseg = tot >> 16;
            int po = ex0 & 0xFFFF, so = ex0 >> 16;
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int idx = kPer * t + u;
                if (c[u] > 0) {
                    S.seg_start[so] = po;
                    bins[idx] = (so << 16) | po;
                    ++so;
                    po += c[u];
                }
            }
            if (t == 0) S.seg_start[nseg] = nact;
            __syncthreads();
            if (act) put_record((bins[key] & 0xFFFF) + rank);
        } else {
            // a CTA spread over too many cells: compact, and let runs of equal
            // base in memory order form the segments
            const int k = block_excl_scan<kScatterChunk>(act ? 1 : 0, &nact);
            if (act) { S.base[0][k] = b0; S.base[1][k] = b1; S.base[2][k] = b2; }
            __syncthreads();
            const bool head = t < nact && (t == 0 || S.base[0][t] != S.base[0][t - 1] ||
                                           S.base[1][t] != S.base[1][t - 1] || S.base[2][t] != S.base[2][t - 1]);
            const int sidx = block_excl_scan<kScatterChunk>(head ? 1 : 0, &nseg);
            if (head) S.seg_start[sidx] = t;
            if (t == 0) S.seg_start[nseg] = nact;
            __syncthreads();
            if (act) put_record(k);
        }
    }
    __syncthreads();  // records and segments complete

    // Work: the items (segment s, stencil column ij = 3i + j), q = 9 s + ij.
    // Complete passes over the threads take whole items: a thread sums its
    // column's particles in registers and adds the column's 3 nodes once.  The
    // items left over (fewer than the threads) get g lanes each (g a power of
    // two, g x items <= threads): the g lanes of an item take its particles
    // strided by g, sum their partial columns with warp shuffles, and one adds
    // the column -- so no two lanes add into the same node at once.
    ColumnSums acc;
    const int items = 9 * nseg;
    const int full_items = (items / kScatterChunk) * kScatterChunk;
    for (int q = t; q < full_items; q += kScatterChunk) {
        const int s = q / 9, ij = q - 9 * s;
        const int i = ij / 3, j = ij - 3 * (ij / 3);
        const float2 fi2 = dup2((float)i), fj2 = dup2((float)j);
        const int k0 = S.seg_start[s], k1 = S.seg_start[s + 1];
        acc.zero();
        for (int kq = k0; kq < k1; ++kq) acc.add(S, scatter_slot(kq), i, j, fi2, fj2);
        acc.emit(S, k0, ij, gmv, nx, ny, nz, bad);
    }
    const int left = items - full_items;  // uniform, < kScatterChunk
    if (left > 0) {
        int lg = 0;
        while (lg < 5 && (left << (lg + 1)) <= kScatterChunk) ++lg;
        const int q = full_items + (t >> lg), sub = t & ((1 << lg) - 1);
        const bool mine = q < items;
        int k0 = 0, ij = 0;
        acc.zero();
        if (mine) {
            const int s = q / 9;
            ij = q - 9 * s;
            k0 = S.seg_start[s];
            const int k1 = S.seg_start[s + 1];
            const int i = ij / 3, j = ij - 3 * (ij / 3);
            const float2 fi2 = dup2((float)i), fj2 = dup2((float)j);
            for (int kq = k0 + sub; kq < k1; kq += 1 << lg) acc.add(S, scatter_slot(kq), i, j, fi2, fj2);
        }
        for (int o = (1 << lg) >> 1; o > 0; o >>= 1) acc.shfl_add(o);  // all lanes (full-warp shuffles)
        if (mine && sub == 0) acc.emit(S, k0, ij, gmv, nx, ny, nz, bad);
    }
}

// One particle's 27-node scatter straight into global memory (rare particles
// handled outside the CTA-cooperative path); same arithmetic per node.
__device__ __forceinline__ void p2g_scatter_one(const float *xp, const float *v, const float *C0, const float *st6,
                                                float m, float vol, const mpmw_params_t &prm,
                                                float4 *__restrict__ gmv, int nx, int ny, int nz, uint32_t &bad)
{
    Weights W;
    weights(xp, prm.min_bounds, prm.inv_dx, W);
    const float r = prm.rpic_damping;
    float Cp[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            Cp[3 * a + b] = (1.f - r) * C0[3 * a + b] + (r / 2.f) * (C0[3 * a + b] - C0[3 * b + a]);
    if (r < -0.001f) {
#pragma unroll
        for (int q = 0; q < 9; ++q) Cp[q] = 0.f;
    }
    const float mdx = m * prm.dx;
    float B[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) B[q] = Cp[q] * mdx;
    float a[3];
#pragma unroll
    for (int row = 0; row < 3; ++row)
        a[row] = fma_(-B[3 * row + 0], W.fx[0], fma_(-B[3 * row + 1], W.fx[1], fma_(-B[3 * row + 2], W.fx[2], m * v[row])));
    const float sc = -(prm.dt * vol) * prm.inv_dx;
    const float s00 = sc * st6[0], s11 = sc * st6[1], s22 = sc * st6[2], s01 = sc * st6[3], s02 = sc * st6[4],
                s12 = sc * st6[5];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const float fi = (float)i, fj = (float)j;
            const float wxy = W.w[0][i] * W.w[1][j], g0 = W.dw[0][i] * W.w[1][j], g1 = W.w[0][i] * W.dw[1][j];
            const float wm = wxy * m;
            const float A0 = fma_(fj, B[1], fma_(fi, B[0], a[0]));
            const float A1 = fma_(fj, B[4], fma_(fi, B[3], a[1]));
            const float A2 = fma_(fj, B[7], fma_(fi, B[6], a[2]));
            const float Q0 = fma_(s00, g0, s01 * g1), Q1 = fma_(s01, g0, s11 * g1), Q2 = fma_(s02, g0, s12 * g1);
            const float R0 = wxy * s02, R1 = wxy * s12, R2 = wxy * s22;
            float P0 = fma_(wxy, A0, Q0), P1 = fma_(wxy, A1, Q1), P2 = fma_(wxy, A2, Q2);
            const float dz0 = wxy * B[2], dz1 = wxy * B[5], dz2 = wxy * B[8];
            const int gx = W.base[0] + i, gy = W.base[1] + j;
            for (int kk = 0; kk < 3; ++kk) {
                if (kk > 0) { P0 = P0 + dz0; P1 = P1 + dz1; P2 = P2 + dz2; }
                const float wz = W.w[2][kk], dwz = W.dw[2][kk];
                const float4 c = make_float4(wz * wm, fma_(wz, P0, dwz * R0), fma_(wz, P1, dwz * R1),
                                             fma_(wz, P2, dwz * R2));
                const int gz = W.base[2] + kk;
                if (gx < 0 || gy < 0 || gz < 0 || gx >= nx || gy >= ny || gz >= nz) { bad |= MPMW_ST_OOB; continue; }
                atomicAdd(&gmv[((int64_t)gx * ny + gy) * nz + gz], c);
            }
        }
}

}  // namespace mpmw
