// mpmw_xpbd.cu -- XPBD substep kernels and the spatial hash (C-ABI entry points).
//
// Reference (MPMWarpYDW): utils/xpbdRoutines.py, launch order
// utils/simulationRoutines.py:295-526, hash grid wp.HashGrid (simStates.py:174).
//
// Spatial hash (restates wp.HashGrid's documented behaviour):
//   cell of a point  = truncating casts of p * (1/cell_width) per axis, offset by
//                      2^20, clamped at 0, reduced modulo the hash dims;
//                      hash = cz*(dx*dy) + cy*dx + cx
//   point order      = stable sort of point indices by hash (LSD radix sort,
//                      7-bit digits, rank within a tile taken in index order)
//   cell ranges      = [start, end) of each hash in the sorted order, 0/0 if empty
//   query            = cells from trunc((p - r)/w) to trunc((p + r)/w) per axis
//                      (at most dims cells per axis), x fastest, then y, then z;
//                      within a cell, sorted order
#include <atomic>
#include <cstring>
#include "mpmw_common.cuh"
#include "mpmw_math.cuh"
#include "mpmw_scan.cuh"
#include "mpmw_gridsync.cuh"
#include "../../include/mpmw_xpbd.h"

namespace mpmw {

// ---------------------------------------------------------------------------
// hash cells
// ---------------------------------------------------------------------------
__device__ __forceinline__ int hash_index(const int *hd, int x, int y, int z)
{
    const int origin = 1 << 20;
    x += origin; y += origin; z += origin;
    x = x < 0 ? 0 : x;
    y = y < 0 ? 0 : y;
    z = z < 0 ? 0 : z;
    int cx = x % hd[0], cy = y % hd[1], cz = z % hd[2];
    return cz * (hd[0] * hd[1]) + cy * hd[0] + cx;
}

struct HashDims { int d[3]; };

__device__ __forceinline__ void hash_cell_at(const float *x, int64_t n, float inv, const HashDims &hd,
                                             int *keys, int *ids,
                                             int *point_cells, int64_t p)
{
    int cx = (int)(x[p] * inv), cy = (int)(x[n + p] * inv), cz = (int)(x[2 * n + p] * inv);
    int h = hash_index(hd.d, cx, cy, cz);
    keys[p] = h;
    ids[p] = (int)p;
    if (point_cells) point_cells[p] = h;
}

__global__ void k_hash_cells(const float *__restrict__ x, int64_t n, float inv, HashDims hd, int *__restrict__ keys,
                             int *__restrict__ ids, int *__restrict__ point_cells)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) hash_cell_at(x, n, inv, hd, keys, ids, point_cells, p);
}

// one bit per hash cell: set where a particle labelled XPBD lies (its cell
// from the same positions and formula as k_hash_cells)
__device__ __forceinline__ void mark_xpbd_cell_at(const mpmw_particles_t &P, float inv, const HashDims &hd,
                                                  unsigned *bits, int64_t p)
{
    const int64_t n = P.n;
    if (P.material[p] != 2) return;
    int cx = (int)(P.x[p] * inv), cy = (int)(P.x[n + p] * inv), cz = (int)(P.x[2 * n + p] * inv);
    int h = hash_index(hd.d, cx, cy, cz);
    atomicOr(&bits[h >> 5], 1u << (h & 31));
}

__global__ void k_mark_xpbd_cells(mpmw_particles_t P, float inv, HashDims hd, unsigned *__restrict__ bits)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P.n) mark_xpbd_cell_at(P, inv, hd, bits, p);
}

// ---------------------------------------------------------------------------
// stable LSD radix sort of (key, id) pairs, 7-bit digits
// ---------------------------------------------------------------------------
constexpr int kRadixBits = 7;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;  // 4096 items per tile

// per-tile digit histogram, stored digit-major: hist[d * ntiles + tile].
// Every thread of a kSortThreads CTA calls it (it synchronizes the block,
// last of all so that the CTA can go on to another tile).
__device__ __forceinline__ void radix_hist_tile(int *h, const int *keys, int64_t n, int shift, int ntiles,
                                                int *hist, int tile)
{
    for (int i = threadIdx.x; i < kRadix; i += blockDim.x) h[i] = 0;
    __syncthreads();
    int64_t base = (int64_t)tile * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        int64_t i = base + (int64_t)r * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadix - 1)], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) hist[(int64_t)d * ntiles + tile] = h[d];
    __syncthreads();
}

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const int *__restrict__ keys, int64_t n, int shift,
                                                            int ntiles, int *__restrict__ hist)
{
    __shared__ int h[kRadix];
    radix_hist_tile(h, keys, n, shift, ntiles, hist, blockIdx.x);
}

constexpr int kSortWarps = kSortThreads / 32;
struct RadixScatterShared {
    int run[kRadix];               // items of each digit placed by earlier rounds
    int wcnt[kSortWarps][kRadix];  // per-warp digit counts of the current round
    int tile_off[kRadix];
};

// stable scatter of one tile: offsets[d * ntiles + tile] is the exclusive
// prefix of hist.  Every thread of a kSortThreads CTA calls it.
__device__ __forceinline__ void radix_scatter_tile(RadixScatterShared &S, const int *kin,
                                                   const int *vin, int64_t n, int shift, int ntiles,
                                                   const int *offsets, int *kout,
                                                   int *vout, int tile)
{
    constexpr int kWarps = kSortWarps;
    int *run = S.run, *tile_off = S.tile_off;
    auto &wcnt = S.wcnt;
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
        run[d] = 0;
        tile_off[d] = offsets[(int64_t)d * ntiles + tile];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int64_t base = (int64_t)tile * kSortTile;
    for (int r = 0; r < kSortRounds; ++r) {
        for (int d = threadIdx.x; d < kWarps * kRadix; d += blockDim.x) (&wcnt[0][0])[d] = 0;
        __syncthreads();
        int64_t i = base + (int64_t)r * kSortThreads + threadIdx.x;
        bool valid = i < n;
        int key = valid ? kin[i] : 0;
        int val = valid ? vin[i] : 0;
        int dig = valid ? ((key >> shift) & (kRadix - 1)) : kRadix;  // invalid items in their own class
        unsigned peers = __match_any_sync(0xffffffffu, dig);
        int rank = __popc(peers & lt);
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) wcnt[wid][dig] = __popc(peers);
        __syncthreads();
        if (valid) {
            int before = 0;
            for (int w = 0; w < wid; ++w) before += wcnt[w][dig];
            int pos = tile_off[dig] + run[dig] + before + rank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        for (int d = threadIdx.x; d < kRadix; d += blockDim.x) {
            int s = 0;
            for (int w = 0; w < kWarps; ++w) s += wcnt[w][d];
            run[d] += s;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const int *__restrict__ kin, const int *__restrict__ vin,
                                                               int64_t n, int shift, int ntiles,
                                                               const int *__restrict__ offsets, int *__restrict__ kout,
                                                               int *__restrict__ vout)
{
    __shared__ RadixScatterShared S;
    radix_scatter_tile(S, kin, vin, n, shift, ntiles, offsets, kout, vout, blockIdx.x);
}

__device__ __forceinline__ void cell_range_at(const int *skeys, int64_t n, int *starts,
                                              int *ends, int64_t i)
{
    int c = skeys[i];
    if (i == 0 || skeys[i - 1] != c) starts[c] = (int)i;
    if (i == n - 1 || skeys[i + 1] != c) ends[c] = (int)(i + 1);
}

__global__ void k_cell_ranges(const int *__restrict__ skeys, int64_t n, int *__restrict__ starts, int *__restrict__ ends)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cell_range_at(skeys, n, starts, ends, i);
}

static int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }

size_t hash_workspace_bytes(int64_t n)
{
    int64_t nt = sort_tiles(n);
    int64_t hist = (int64_t)kRadix * nt;
    int64_t scan_scratch = scan_blocks(hist > 0 ? hist : 1) + 1;
    // keys_a, keys_b, ids_b, hist, offsets, scan scratch (ints), 256-byte aligned pieces
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    return (size_t)(al(4 * n) * 3 + al(4 * hist) * 2 + al(4 * scan_scratch));
}

// Stable LSD radix sort of the (key, id) pairs in keys_a / ids_a over the low
// `bits` bits of the keys, with the workspace carved as hash_workspace_bytes
// lays it out after those two arrays; returns the arrays that hold the sorted
// pairs (either the a or the b buffers) in *keys_out / *ids_out.
static int radix_sort_pairs(int *keys_a, int *ids_a, int64_t n, int bits, char *w, int **keys_out, int **ids_out,
                            cudaStream_t s)
{
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    const int64_t nt = sort_tiles(n), hist_n = (int64_t)kRadix * nt;
    int *keys_b = reinterpret_cast<int *>(w); w += al(4 * n);
    int *ids_b = reinterpret_cast<int *>(w); w += al(4 * n);
    int *hist = reinterpret_cast<int *>(w); w += al(4 * hist_n);
    int *offs = reinterpret_cast<int *>(w); w += al(4 * hist_n);
    int *scr = reinterpret_cast<int *>(w);
    int *ki = keys_a, *vi = ids_a, *ko = keys_b, *vo = ids_b;
    for (int shift = 0; shift < bits; shift += kRadixBits) {
        k_radix_hist<<<(unsigned)nt, kSortThreads, 0, s>>>(ki, n, shift, (int)nt, hist);
        MPMW_TRY_LAUNCH("k_radix_hist");
        if (!exclusive_scan(hist, offs, hist_n, scr, s)) { set_error("radix sort: too many items"); return MPMW_E_ARG; }
        MPMW_TRY_LAUNCH("scan");
        k_radix_scatter<<<(unsigned)nt, kSortThreads, 0, s>>>(ki, vi, n, shift, (int)nt, offs, ko, vo);
        MPMW_TRY_LAUNCH("k_radix_scatter");
        int *t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    *keys_out = ki;
    *ids_out = vi;
    return MPMW_OK;
}

// Key of the 4x4x4-cell block order (block = edge in cells): the particle's
// stencil base cell int((x - min_bounds) inv_dx - 0.5) per axis (truncation,
// utils/mpmRoutines.py:514-517), clamped to the grid, as
// (block index, C order) * block^3 + (cell within the block, C order).
__global__ void k_block_keys(const float *__restrict__ x, int64_t n, float mb0, float mb1, float mb2, float inv_dx,
                             int d0, int d1, int d2, int block, int *__restrict__ keys, int *__restrict__ ids)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float mb[3] = {mb0, mb1, mb2};
    const int d[3] = {d0, d1, d2};
    int c[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float gp = (x[(int64_t)a * n + p] - mb[a]) * inv_dx;
        const float f = gp - 0.5f;
        // truncation toward zero of a finite value; non-finite or huge positions clamp
        int v = isfinite(f) ? (f >= 2.0e9f ? INT32_MAX : (f <= -2.0e9f ? INT32_MIN : (int)f)) : 0;
        v = v < 0 ? 0 : v;
        c[a] = v > d[a] - 1 ? d[a] - 1 : v;
    }
    const int nb1 = (d1 + block - 1) / block, nb2 = (d2 + block - 1) / block;
    const int bidx = ((c[0] / block) * nb1 + c[1] / block) * nb2 + c[2] / block;
    const int ridx = ((c[0] % block) * block + c[1] % block) * block + c[2] % block;
    keys[p] = bidx * (block * block * block) + ridx;
    ids[p] = (int)p;
}

// the block keys, then the radix sort's buffers: the hash build's layout
size_t block_sort_workspace_bytes(int64_t n) { return hash_workspace_bytes(n); }

int block_sort(const float *x, int64_t n, const mpmw_params_t &prm, const int32_t *dims, int block, int32_t *perm,
               void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (ws_bytes < block_sort_workspace_bytes(n)) {
        set_error("block_sort: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  block_sort_workspace_bytes(n));
        return MPMW_E_WORKSPACE;
    }
    if (n == 0) return MPMW_OK;
    const int64_t nb = (int64_t)((dims[0] + block - 1) / block) * ((dims[1] + block - 1) / block) *
                       ((dims[2] + block - 1) / block);
    const int64_t nkeys = nb * block * block * block;
    if (nkeys > (int64_t)INT32_MAX) {
        set_error("block_sort: %lld block keys exceed the 31-bit key range", (long long)nkeys);
        return MPMW_E_ARG;
    }
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    char *w = static_cast<char *>(ws);
    int *keys_a = reinterpret_cast<int *>(w); w += al(4 * n);
    k_block_keys<<<grid_for(n), kBlock, 0, s>>>(x, n, prm.min_bounds[0], prm.min_bounds[1], prm.min_bounds[2],
                                                prm.inv_dx, dims[0], dims[1], dims[2], block, keys_a, perm);
    MPMW_TRY_LAUNCH("k_block_keys");
    int bits = 0;
    for (int64_t c = nkeys - 1; c > 0; c >>= 1) ++bits;
    int *ko = nullptr, *vo = nullptr;
    int rc = radix_sort_pairs(keys_a, perm, n, bits, w, &ko, &vo, s);
    if (rc != MPMW_OK) return rc;
    if (vo != perm && cudaMemcpyAsync(perm, vo, n * sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
        set_error("block_sort: copy failed");
        return MPMW_E_DEVICE;
    }
    return MPMW_OK;
}

int hash_build(const float *x, int64_t n, const mpmw_hash_t &h, void *ws, size_t ws_bytes, cudaStream_t s)
{
    if (ws_bytes < hash_workspace_bytes(n)) {
        set_error("hash_build: workspace of %zu bytes is smaller than the %zu required", ws_bytes,
                  hash_workspace_bytes(n));
        return MPMW_E_WORKSPACE;
    }
    const int64_t ncell = (int64_t)h.dims[0] * h.dims[1] * h.dims[2];
    if (cudaMemsetAsync(h.cell_starts, 0, ncell * sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(h.cell_ends, 0, ncell * sizeof(int), s) != cudaSuccess) {
        set_error("hash_build: memset failed");
        return MPMW_E_DEVICE;
    }
    if (n == 0) return MPMW_OK;
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    char *w = static_cast<char *>(ws);
    int *keys_a = reinterpret_cast<int *>(w); w += al(4 * n);
    int *ids_a = h.point_ids;  // the sorted ids end up here (3 passes: a->b->a->b, then copy)
    HashDims hd{{h.dims[0], h.dims[1], h.dims[2]}};
    float inv = 1.0f / h.cell_width;
    k_hash_cells<<<grid_for(n), kBlock, 0, s>>>(x, n, inv, hd, keys_a, ids_a, h.point_cells);
    MPMW_TRY_LAUNCH("k_hash_cells");
    int bits = 0;
    for (int64_t c = ncell - 1; c > 0; c >>= 1) ++bits;
    int *ki = nullptr, *vi = nullptr;
    {
        int rc = radix_sort_pairs(keys_a, ids_a, n, bits, w, &ki, &vi, s);
        if (rc != MPMW_OK) return rc;
    }
    if (vi != h.point_ids) {
        if (cudaMemcpyAsync(h.point_ids, vi, n * sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
            set_error("hash_build: copy failed");
            return MPMW_E_DEVICE;
        }
    }
    k_cell_ranges<<<grid_for(n), kBlock, 0, s>>>(ki, n, h.cell_starts, h.cell_ends);
    MPMW_TRY_LAUNCH("k_cell_ranges");
    return MPMW_OK;
}

// ---------------------------------------------------------------------------
// XPBD kernels
// ---------------------------------------------------------------------------
// copies (x, v) into the integrated buffers and integrates XPBD particles
// (simulationRoutines.py:314-331 + xpbdRoutines.py:23-48)
// flag bit0: read from the particle x/v (else from x_int/v_int);
// flag bit1: write every particle (the wp.copy), else only integrated ones.
// xpbd_count (optional, zeroed by the caller): receives the number of
// particles labelled XPBD, active or not.
__device__ __forceinline__ void xpbd_integrate_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int flag,
                                 int *xpbd_count = nullptr)
{
    const int64_t n = P.n;
    const int mat = p < n ? P.material[p] : 0;
    const bool integ = p < n && P.active[p] == 1 && mat == 2;
    if (xpbd_count) {
        const unsigned m = __ballot_sync(0xffffffffu, mat == 2);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(xpbd_count, __popc(m));
    }
    if (p >= n) return;
    float x0[3], v0[3];
    load3((flag & 1) ? P.x : X.x_int, n, p, x0);
    load3((flag & 1) ? P.v : X.v_int, n, p, v0);
    if (integ) {
        float v1[3] = {v0[0] + q.gravity[0] * q.dt, v0[1] + q.gravity[1] * q.dt, v0[2] + q.gravity[2] * q.dt};
        float m = len3(v1);
        if (m > q.v_max) { float s = q.v_max / m; v1[0] = v1[0] * s; v1[1] = v1[1] * s; v1[2] = v1[2] * s; }
#pragma unroll
        for (int a = 0; a < 3; ++a) { x0[a] = x0[a] + v1[a] * q.dt; v0[a] = v1[a]; }
    }
    if (integ || (flag & 2)) {
        store3(X.x_int, n, p, x0);
        store3(X.v_int, n, p, v0);
    }
}

__global__ void k_xpbd_integrate(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int flag,
                                 int *xpbd_count = nullptr)
{
    xpbd_integrate_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q, flag, xpbd_count);
}

// xpbdRoutines.py:3-21
__device__ __forceinline__ void reset_labels_at(int64_t p, mpmw_particles_t P)
{
    if (p >= P.n) return;
    if (P.active[p] == 1 && P.material[p] == 0) P.material[p] = 1;
}

__global__ void k_reset_labels(mpmw_particles_t P)
{
    reset_labels_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P);
}

// xpbdRoutines.py:49-136; writes delta (the reference zeroes it first, then adds)
__device__ __forceinline__ void bound_contacts_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int accumulate)
{
    const int64_t n = P.n;
    if (p >= n) return;
    float acc[3] = {0.f, 0.f, 0.f};
    if (accumulate) load3(X.delta, n, p, acc);
    if (P.active[p] == 1 && P.material[p] == 2 && P.mass[p] != 0.f) {
        float wi = 1.f / P.mass[p];
        float xp[3], vp[3];
        load3(X.x_int, n, p, xp);
        load3(X.v_int, n, p, vp);
        float r = P.radius[p];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                float nrm[3] = {0.f, 0.f, 0.f};
                nrm[i] = side == 0 ? 1.f : -1.f;
                const float *b = side == 0 ? q.bmin : q.bmax;
                float d[3] = {xp[0] - b[0], xp[1] - b[1], xp[2] - b[2]};
                float c = rmin(dot3(nrm, d) - r, 0.f);
                if (!(c < 0.f)) continue;
                float ln = c;
                float dn[3] = {nrm[0] * ln, nrm[1] * ln, nrm[2] * ln};
                float vn = dot3(nrm, vp);
                float fmu = q.dyn_friction;
                if (fabsf(vn) < q.static_thr * r) fmu = q.static_friction;
                float vt[3] = {vp[0] - nrm[0] * vn, vp[1] - nrm[1] * vn, vp[2] - nrm[2] * vn};
                float vtl = len3(vt);
                float lf = rmax(fmu * ln, -vtl * q.dt);
                float df[3] = {0.f, 0.f, 0.f};
                if (vtl > 1e-8f) { float nv[3]; normalize3(vt, nv); df[0] = nv[0] * lf; df[1] = nv[1] * lf; df[2] = nv[2] * lf; }
#pragma unroll
                for (int a = 0; a < 3; ++a) acc[a] = acc[a] + (((df[a] - dn[a]) / wi) * q.relaxation) * wi;
            }
        }
    }
    store3(X.delta, n, p, acc);
}

__global__ void k_bound_contacts(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int accumulate)
{
    bound_contacts_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q, accumulate);
}

// xpbdRoutines.py:138-219.  One thread per sorted position tid; the outer
// checks use tid, the work uses the sorted point i (reference behaviour).
// Each deltas[i] is owned by exactly one thread, so it is read-modify-written
// without atomics; the contact-lock label writes only ever store 0 over a
// label <= 1, which no test in this kernel distinguishes from 1.
// xpbd_count (optional): the step's number of particles labelled XPBD.  Every
// pair this kernel acts on has an XPBD-labelled particle in it (the working
// particle i may be an inactive one: the activity test is on tid), so with
// none there is nothing to do: each particle's loop would add +0 to a delta
// that k_bound_contacts left at +0, and set no label.
// xpbd_cells (optional): one bit per hash cell holding an XPBD-labelled
// particle.  A non-XPBD particle whose query box has no such cell has no pair
// to act on and returns before walking its neighbours (same argument).
// Rec: the neighbours' fields come from per-sorted-slot records
// (k_contact_records) instead of by point index from the particle arrays.
// The records hold the same values (labels as of the kernel's start, which the
// tests here cannot tell from the live ones: the lock only writes 0 over <= 1).
template <bool Rec>
__device__ __forceinline__ void particle_contacts_at(int64_t tid, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_hash_t H, mpmw_xpbd_params_t q,
                                    const int *xpbd_count = nullptr, const unsigned *xpbd_cells = nullptr,
                                    const float4 *recA = nullptr,
                                    const float4 *recB = nullptr)
{
    const int64_t n = P.n;
    if (tid >= n) return;
    if (xpbd_count && *(xpbd_count) == 0) return;
    if (P.active[tid] != 1) return;
    if (!(P.material[tid] >= 0)) return;
    int i = H.point_ids[tid];
    if (i == -1) return;
    float xi[3], vi[3];
    load3(X.x_int, n, i, xi);
    load3(X.v_int, n, i, vi);
    float rad = P.radius[i];
    if (P.mass[tid] == 0.f) return;
    float w1 = 1.f / P.mass[i];
    const float inv = 1.0f / H.cell_width;
    const float qr = (rad + q.max_radius) + q.cohesion * rad;
    const int hd[3] = {H.dims[0], H.dims[1], H.dims[2]};
    int xs = (int)((xi[0] - qr) * inv), ys = (int)((xi[1] - qr) * inv), zs = (int)((xi[2] - qr) * inv);
    int xe = (int)((xi[0] + qr) * inv), ye = (int)((xi[1] + qr) * inv), ze = (int)((xi[2] + qr) * inv);
    xe = xe < xs + hd[0] - 1 ? xe : xs + hd[0] - 1;
    ye = ye < ys + hd[1] - 1 ? ye : ys + hd[1] - 1;
    ze = ze < zs + hd[2] - 1 ? ze : zs + hd[2] - 1;
    float dl[3] = {0.f, 0.f, 0.f};
    const float alpha = 0.f;
    float k_mu = q.dyn_friction;
    int mat_i = P.material[i];
    if (xpbd_cells && mat_i <= 1) {
        bool any = false;
        for (int cz = zs; cz <= ze && !any; ++cz)
            for (int cy = ys; cy <= ye && !any; ++cy)
                for (int cx = xs; cx <= xe && !any; ++cx) {
                    const int c = hash_index(hd, cx, cy, cz);
                    any = (xpbd_cells[c >> 5] >> (c & 31)) & 1u;
                }
        if (!any) return;
    }
    // one candidate pair (i, index) that passed the activity and label tests
    auto pair = [&](int index, int mat_j, const float *xj, float rad_j, float mass_j) {
        float nn[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
        float d = len3(nn);
        float err = (d - rad) - rad_j;
        float w2 = 1.f / mass_j;
        float denom = w1 + w2;
        if (err <= q.cohesion && denom > 0.f) {
            if (q.lock == 1) {
                if (mat_i <= 1 && mat_j == 2) P.material[i] = 0;
                if (mat_i == 2 && mat_j <= 1) P.material[index] = 0;
            }
            float nu[3] = {nn[0] / d, nn[1] / d, nn[2] / d};
            float vj[3];
            load3(X.v_int, n, index, vj);
            float vrel[3] = {vi[0] - vj[0], vi[1] - vj[1], vi[2] - vj[2]};
            float ln = err / (1.f + (alpha * q.dt) * q.dt);
            float dn[3] = {nu[0] * ln, nu[1] * ln, nu[2] * ln};
            float vn = dot3(nu, vrel);
            if (fabsf(vn) < q.static_thr * rad) k_mu = q.static_friction;
            float vt[3] = {vrel[0] - nu[0] * vn, vrel[1] - nu[1] * vn, vrel[2] - nu[2] * vn};
            float lf = rmax(k_mu * ln, -len3(vt) * q.dt);
            float nv[3];
            normalize3(vt, nv);
            float df[3] = {nv[0] * lf, nv[1] * lf, nv[2] * lf};
#pragma unroll
            for (int a = 0; a < 3; ++a) dl[a] = dl[a] + ((df[a] - dn[a]) / denom) * w1;
        }
    };
    // The walk visits the query box's cells x fastest, then y, then z, and
    // each cell's slots in sorted order.
    if constexpr (Rec) {
        // One item ahead: the next cell's slot range and the next record are
        // loaded before the current record is used, so their latencies overlap.
        const int nqx = xe - xs + 1, nqy = ye - ys + 1, nqz = ze - zs + 1;
        const int nq = (nqx > 0 && nqy > 0 && nqz > 0) ? nqx * nqy * nqz : 0;
        int qx = 0, qy = 0, qz = 0;  // the next cell of the walk (offsets in the box)
        int nb = 0, ne = 0;          // its slot range
        auto next_range = [&]() {
            const int c = hash_index(hd, xs + qx, ys + qy, zs + qz);
            nb = H.cell_starts[c];
            ne = H.cell_ends[c];
            if (++qx == nqx) { qx = 0; if (++qy == nqy) { qy = 0; ++qz; } }
        };
        float4 pa = make_float4(0.f, 0.f, 0.f, 0.f), pb = pa;
        int pre = -1;  // slot whose record pa, pb hold
        if (nq > 0) next_range();
        for (int kq = 0; kq < nq; ++kq) {
            const int b = nb, e = ne;
            if (kq + 1 < nq) next_range();
            else nb = ne = 0;
            if (b < e && pre != b) { pa = recA[b]; pb = recB[b]; pre = b; }
            for (int s = b; s < e; ++s) {
                const float4 ra = pa, rb = pb;
                // the following record: this cell's next slot, or the next cell's first
                const int sn = s + 1 < e ? s + 1 : (nb < ne ? nb : -1);
                if (sn >= 0) { pa = recA[sn]; pb = recB[sn]; pre = sn; }
                const int index = __float_as_int(rb.w);
                const float mass_j = rb.x;
                if (!(__float_as_int(rb.y) == 1 && index != i && mass_j > 0.f)) continue;
                const int mat_j = __float_as_int(rb.z);
                if (mat_i <= 1 && mat_j <= 1) continue;
                const float xj[3] = {ra.x, ra.y, ra.z};
                pair(index, mat_j, xj, ra.w, mass_j);
            }
        }
    } else {
        for (int cz = zs; cz <= ze; ++cz)
            for (int cy = ys; cy <= ye; ++cy)
                for (int cx = xs; cx <= xe; ++cx) {
                    const int c = hash_index(hd, cx, cy, cz);
                    const int b = H.cell_starts[c], e = H.cell_ends[c];
                    for (int s = b; s < e; ++s) {
                        const int index = H.point_ids[s];
                        if (!(P.active[index] == 1 && index != i && P.mass[index] > 0.f)) continue;
                        const int mat_j = P.material[index];
                        if (mat_i <= 1 && mat_j <= 1) continue;
                        float xj[3];
                        load3(X.x_int, n, index, xj);
                        pair(index, mat_j, xj, P.radius[index], P.mass[index]);
                    }
                }
    }
    float cur[3];
    load3(X.delta, n, i, cur);
#pragma unroll
    for (int a = 0; a < 3; ++a) cur[a] = cur[a] + dl[a] * q.relaxation;
    store3(X.delta, n, i, cur);
}

template <bool Rec>
__global__ void __launch_bounds__(kBlock, 4) k_particle_contacts(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_hash_t H, mpmw_xpbd_params_t q,
                                    const int *xpbd_count = nullptr, const unsigned *xpbd_cells = nullptr,
                                    const float4 *__restrict__ recA = nullptr,
                                    const float4 *__restrict__ recB = nullptr)
{
    particle_contacts_at<Rec>((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, H, q, xpbd_count, xpbd_cells, recA, recB);
}

// The fields the contact pass reads of its neighbours, one record per sorted
// hash slot s (point i = point_ids[s]): (x_int, radius) and (mass, active,
// material, i), so a neighbour walk reads contiguous memory in hash order.
// Nothing to write when the step has no XPBD-labelled particle (xpbd_count):
// the contact pass then reads no record.
__device__ __forceinline__ void contact_records_at(int64_t s, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_hash_t H, float4 *recA,
                                  float4 *recB, const int *xpbd_count)
{
    const int64_t n = P.n;
    if (s >= n) return;
    if (xpbd_count && *(xpbd_count) == 0) return;
    const int i = H.point_ids[s];
    if (i < 0 || i >= n) {
        recA[s] = make_float4(0.f, 0.f, 0.f, 0.f);
        recB[s] = make_float4(0.f, __int_as_float(0), __int_as_float(0), __int_as_float(-1));
        return;
    }
    float x[3];
    load3(X.x_int, n, i, x);
    recA[s] = make_float4(x[0], x[1], x[2], P.radius[i]);
    recB[s] = make_float4(P.mass[i], __int_as_float(P.active[i]), __int_as_float(P.material[i]), __int_as_float(i));
}

__global__ void k_contact_records(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_hash_t H, float4 *__restrict__ recA,
                                  float4 *__restrict__ recB, const int *xpbd_count)
{
    contact_records_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, H, recA, recB, xpbd_count);
}

// xpbdRoutines.py:221-257 my_apply_particle_deltas.  x_orig = particle x,
// x_pred = x_int.  flag 0/1 (substep): the surrounding copies
// (simulationRoutines.py:398-421) are folded in -- x_int/v_int are updated in
// place, and with flag 1 the deltaInt buffers receive the same values for every
// particle.  flag 2 (the kernel alone): results go to x_dI/v_dI for active
// particles only, x_int/v_int are left untouched.
__device__ __forceinline__ void apply_deltas_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int flag)
{
    const int64_t n = P.n;
    if (p >= n) return;
    float xn[3], vn[3];
    load3(X.x_int, n, p, xn);
    if (flag != 2) load3(X.v_int, n, p, vn);
    const bool act = P.active[p] == 1;
    if (act) {
        float d[3];
        load3(X.delta, n, p, d);
        if (isnan(d[0]) || isnan(d[1]) || isnan(d[2])) d[0] = d[1] = d[2] = 0.f;
        float x0[3];
        load3(P.x, n, p, x0);
#pragma unroll
        for (int a = 0; a < 3; ++a) { xn[a] = xn[a] + d[a]; vn[a] = (xn[a] - x0[a]) / q.dt; }
        float m = len3(vn);
        if (m > q.v_max) { float s = q.v_max / m; vn[0] = vn[0] * s; vn[1] = vn[1] * s; vn[2] = vn[2] * s; }
        if (flag != 2) {
            store3(X.x_int, n, p, xn);
            store3(X.v_int, n, p, vn);
        }
    }
    if (flag == 1 || (flag == 2 && act)) {
        store3(X.x_dI, n, p, xn);
        store3(X.v_dI, n, p, vn);
    }
}

__global__ void k_apply_deltas(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int flag)
{
    apply_deltas_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q, flag);
}

// xpbdRoutines.py:312-334 sleepParticles (counts[0] total, counts[1] sleeping)
__device__ __forceinline__ void sleep_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q)
{
    const int64_t n = P.n;
    bool is = p < n && P.active[p] == 1 && P.material[p] == 2;
    bool slept = false;
    if (is) {
        float a[3], b[3];
        load3(P.x, n, p, b);
        load3(X.x_int, n, p, a);
        float dd[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        float d = len3(dd);
        if (d / q.dt < q.sleep_thr * P.radius[p]) {
            store3(X.x_int, n, p, b);
            slept = true;
        }
        X.cum_dist[p] = X.cum_dist[p] + d;
    }
    // warp-aggregated counters
    unsigned m_all = __ballot_sync(0xffffffffu, is), m_sl = __ballot_sync(0xffffffffu, slept);
    if ((threadIdx.x & 31) == 0 && X.counts) {
        if (m_all) atomicAdd(&X.counts[0], __popc(m_all));
        if (m_sl) atomicAdd(&X.counts[1], __popc(m_sl));
    }
}

__global__ void k_sleep(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q)
{
    sleep_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q);
}

// apply_mpm_contact_impulses (xpbdRoutines.py:259-310): x_orig/v_orig = particle
// x/v, x_final = x_int, v_out = v_int.  With commit (the substep,
// simulationRoutines.py:444-470) v_before_contact <- v first and x <- x_int,
// v <- v_int after.
__device__ __forceinline__ void impulses_commit_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int commit)
{
    const int64_t n = P.n;
    if (p >= n) return;
    float x0[3], v0[3], xf[3], vf[3];
    load3(P.x, n, p, x0);
    load3(P.v, n, p, v0);
    load3(X.x_int, n, p, xf);
    load3(X.v_int, n, p, vf);
    if (commit && X.v_before) store3(X.v_before, n, p, v0);
    if (!commit && !(P.active[p] == 1 && P.material[p] <= 1)) return;
    if (P.active[p] == 1 && P.material[p] <= 1) {
        xf[0] = x0[0]; xf[1] = x0[1]; xf[2] = x0[2];
        if (q.xpbd_only == 0) {
            float vc[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) vc[a] = v0[a] + ((xf[a] - x0[a]) / q.dt) * q.coupling;
            float m = len3(vc);
            if (m > q.v_max) { float s = q.v_max / m; vc[0] = vc[0] * s; vc[1] = vc[1] * s; vc[2] = vc[2] * s; }
            vf[0] = vc[0]; vf[1] = vc[1]; vf[2] = vc[2];
        }
        store3(X.x_int, n, p, xf);
        if (q.xpbd_only == 0) store3(X.v_int, n, p, vf);
    }
    if (commit) {
        store3(P.x, n, p, xf);
        store3(P.v, n, p, vf);
    }
}

__global__ void k_impulses_commit(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q, int commit)
{
    impulses_commit_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q, commit);
}

// xpbdRoutines.py:354-375 swellParticlesType2
__device__ __forceinline__ void swell_at(int64_t p, mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q)
{
    const int64_t n = P.n;
    if (p >= n) return;
    if (P.active[p] != 1 || P.material[p] != 2) return;
    float x[3], x0[3];
    load3(P.x, n, p, x);
    load3(P.x_pc, n, p, x0);
    float dd[3] = {x[0] - x0[0], x[1] - x0[1], x[2] - x0[2]};
    float br = X.base_radius[p];
    float dxv = len3(dd) * br;
    float factor = q.swell_act * br;
    float fmax = q.swell_max * br;
    if (dxv > factor) {
        float sr = X.max_radius[p];
        float nr = br + ((sr - br) * (dxv - factor)) / (fmax - factor);
        nr = rmin(rmax(nr, P.radius[p]), sr);
        P.radius[p] = nr;
    }
}

__global__ void k_swell(mpmw_particles_t P, mpmw_xpbd_t X, mpmw_xpbd_params_t q)
{
    swell_at((int64_t)blockIdx.x * blockDim.x + threadIdx.x, P, X, q);
}


// ---------------------------------------------------------------------------
// The XPBD step as one persistent kernel (cooperative launch: every CTA of the
// grid is resident at once).  Phases are separated by grid barriers; within a
// phase each CTA takes elements (or sort tiles) strided by the grid, and each
// element runs the same device function as the multi-launch step, so the two
// forms give the same bits.
// ---------------------------------------------------------------------------
constexpr int kPersistThreads = kSortThreads;                     // 256
constexpr int kPersistMaxCtas = 4000;                              // chunk sums of the in-kernel scan
constexpr size_t kPersistHeaderBytes = 16384;                      // arrival counter, XPBD count, tile tickets, chunk sums

struct PersistArgs {
    mpmw_particles_t P;
    mpmw_xpbd_t X;
    mpmw_hash_t H;
    mpmw_xpbd_params_t q, qi;  // step parameters; those of the iterations (no lock in XPBD-only steps)
    HashDims hd;
    float inv;                 // 1 / cell width
    int64_t ncell;
    int64_t bit_words;         // words of the per-cell XPBD bits (0: no bits)
    int passes, ntiles;        // radix passes (7 bits each), sort tiles
    int64_t hist_n;            // kRadix * ntiles
    int *keys_a, *keys_b, *ids_scratch, *hist, *offs;
    int *chunk_sums;           // one per CTA
    unsigned *arrive;
    unsigned *tickets;         // contact-pass tiles drawn so far (all iterations)
    int *xpbd_count;
    unsigned *xpbd_cells;
    float4 *recA, *recB;
    uint32_t *status;
    int reset_labels;
};

union PersistShared {
    int h[kRadix];
    RadixScatterShared sc;
};

__device__ __forceinline__ bool persist_scan(const PersistArgs &A, int *s_ok)
{
    const int64_t L = (A.hist_n + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * L;
    const int64_t c1 = c0 + L < A.hist_n ? c0 + L : A.hist_n;
    int part = 0, total = 0;
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) part += A.hist[i];
    block_excl_scan<kPersistThreads>(part, &total);
    if (threadIdx.x == 0) A.chunk_sums[blockIdx.x] = total;
    if (!grid_sync(A.arrive, A.status, s_ok)) return false;
    part = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) part += A.chunk_sums[k];
    int prefix = 0;
    block_excl_scan<kPersistThreads>(part, &prefix);
    for (int64_t b = c0; b < c1; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const int v = i < c1 ? A.hist[i] : 0;
        int tot = 0;
        const int ex = block_excl_scan<kPersistThreads>(v, &tot);
        if (i < c1) A.offs[i] = prefix + ex;
        prefix += tot;
    }
    return grid_sync(A.arrive, A.status, s_ok);
}

// utils/simulationRoutines.py:295-526 in one launch: hash build (keys, radix
// passes, cell ranges), XPBD cell bits, integration, label reset, the Jacobi
// iterations (bound contacts and contact records; particle contacts; apply),
// then sleeping, impulses with the commit, and swelling.
__global__ void __launch_bounds__(kPersistThreads) k_xpbd_step_persistent(const __grid_constant__ PersistArgs A)
{
    __shared__ PersistShared sh;
    __shared__ int s_ok, s_tile;
    const int64_t n = A.P.n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t b0 = (int64_t)blockIdx.x * blockDim.x;  // a CTA-uniform loop start, so warp votes see full warps
    // the sorted ids end in point_ids after the last pass
    int *ids0 = (A.passes & 1) ? A.ids_scratch : A.H.point_ids;
    {
        const int64_t m0 = n > A.ncell ? n : A.ncell;
        const int64_t m = m0 > A.bit_words ? m0 : A.bit_words;
        for (int64_t b = b0; b < m; b += stride) {
            const int64_t e = b + threadIdx.x;
            if (e < A.ncell) { A.H.cell_starts[e] = 0; A.H.cell_ends[e] = 0; }
            if (e < A.bit_words) A.xpbd_cells[e] = 0u;
            if (e < n) hash_cell_at(A.P.x, n, A.inv, A.hd, A.keys_a, ids0, A.H.point_cells, e);
        }
    }
    if (!grid_sync(A.arrive, A.status, &s_ok)) return;
    int *ki = A.keys_a, *vi = ids0, *ko = A.keys_b, *vo = (A.passes & 1) ? A.H.point_ids : A.ids_scratch;
    for (int pass = 0; pass < A.passes; ++pass) {
        const int shift = pass * kRadixBits;
        for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) radix_hist_tile(sh.h, ki, n, shift, A.ntiles, A.hist, t);
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        if (!persist_scan(A, &s_ok)) return;
        for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x)
            radix_scatter_tile(sh.sc, ki, vi, n, shift, A.ntiles, A.offs, ko, vo, t);
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        int *tk = ki; ki = ko; ko = tk;
        int *tv = vi; vi = vo; vo = tv;
    }
    for (int64_t b = b0; b < n; b += stride) {
        const int64_t p = b + threadIdx.x;
        if (p < n) {
            cell_range_at(ki, n, A.H.cell_starts, A.H.cell_ends, p);
            if (A.bit_words) mark_xpbd_cell_at(A.P, A.inv, A.hd, A.xpbd_cells, p);
        }
        xpbd_integrate_at(p, A.P, A.X, A.q, 3, A.xpbd_count);
        if (A.reset_labels) reset_labels_at(p, A.P);
    }
    if (!grid_sync(A.arrive, A.status, &s_ok)) return;
    const int iters = A.qi.iterations;
    for (int it = 0; it < iters; ++it) {
        for (int64_t p = b0 + threadIdx.x; p < n; p += stride) {
            bound_contacts_at(p, A.P, A.X, A.qi, 0);
            contact_records_at(p, A.P, A.X, A.H, A.recA, A.recB, A.xpbd_count);
        }
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        // the neighbour walks vary in length: tiles are handed out as CTAs free up
        const int ctiles = (int)((n + blockDim.x - 1) / blockDim.x);
        const unsigned base = (unsigned)it * (unsigned)(ctiles + (int)gridDim.x);
        for (int t = draw_tile(A.tickets, base, &s_tile); t < ctiles; t = draw_tile(A.tickets, base, &s_tile))
            particle_contacts_at<true>((int64_t)t * blockDim.x + threadIdx.x, A.P, A.X, A.H, A.qi, A.xpbd_count,
                                       A.xpbd_cells, A.recA, A.recB);
        if (!grid_sync(A.arrive, A.status, &s_ok)) return;
        for (int64_t p = b0 + threadIdx.x; p < n; p += stride) apply_deltas_at(p, A.P, A.X, A.qi, it == iters - 1);
        if (it < iters - 1 && !grid_sync(A.arrive, A.status, &s_ok)) return;
    }
    // each particle's own values only from here on (its thread applied its deltas)
    for (int64_t b = b0; b < n; b += stride) {
        const int64_t p = b + threadIdx.x;
        sleep_at(p, A.P, A.X, A.q);
        impulses_commit_at(p, A.P, A.X, A.q, 1);
        if (A.q.swelling_ratio > 0.f) swell_at(p, A.P, A.X, A.q);
    }
}

}  // namespace mpmw

using namespace mpmw;

static int check_xpbd_args(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_xpbd_params_t *q)
{
    if (!p || !x || !q) { set_error("xpbd: NULL argument"); return MPMW_E_ARG; }
    if (p->n < 0) { set_error("xpbd: negative particle count"); return MPMW_E_ARG; }
    if (count_too_large(p->n, "xpbd")) return MPMW_E_ARG;
    if (p->n == 0) return MPMW_OK;
    if (!p->x || !p->v || !p->active || !p->material || !p->mass || !p->radius) {
        set_error("xpbd: x, v, active, material, mass and radius are required");
        return MPMW_E_ARG;
    }
    if (!x->x_int || !x->v_int || !x->delta) { set_error("xpbd: x_int, v_int and delta are required"); return MPMW_E_ARG; }
    if (q->dt == 0.f) { set_error("xpbd: dt must be nonzero"); return MPMW_E_ARG; }
    return MPMW_OK;
}

static int check_hash(const mpmw_hash_t *h, int64_t n)
{
    if (!h) { set_error("hash: NULL"); return MPMW_E_ARG; }
    if (h->dims[0] <= 0 || h->dims[1] <= 0 || h->dims[2] <= 0 ||
        (int64_t)h->dims[0] * h->dims[1] * h->dims[2] > (int64_t)INT32_MAX) {
        set_error("hash: bad dims"); return MPMW_E_ARG;
    }
    if (!(h->cell_width > 0.f)) { set_error("hash: cell_width must be positive"); return MPMW_E_ARG; }
    if (n > 0 && (!h->point_ids || !h->cell_starts || !h->cell_ends)) { set_error("hash: arrays are required"); return MPMW_E_ARG; }
    if (n > (int64_t)INT32_MAX) { set_error("hash: too many points"); return MPMW_E_ARG; }
    return MPMW_OK;
}

#define TRY(expr) do { int _rc = (expr); if (_rc != MPMW_OK) return _rc; } while (0)

extern "C" {

size_t mpmw_hash_workspace_bytes(int64_t n) { return mpmw::hash_workspace_bytes(n < 0 ? 0 : n); }

size_t mpmw_block_sort_workspace_bytes(int64_t n) { return mpmw::block_sort_workspace_bytes(n < 0 ? 0 : n); }

int mpmw_block_sort(const float *x, int64_t n, const mpmw_params_t *prm, const int32_t *dims, int block,
                    int32_t *perm, void *workspace, size_t ws_bytes, mpmw_stream_t stream)
{
    if (count_too_large(n, "block_sort")) return MPMW_E_ARG;
    if (n < 0 || !prm || !dims || block < 1 || block > 16 || (n > 0 && (!x || !perm || !workspace))) {
        set_error("block_sort: bad arguments");
        return MPMW_E_ARG;
    }
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) { set_error("block_sort: grid dims must be positive"); return MPMW_E_ARG; }
    return mpmw::block_sort(x, n, *prm, dims, block, perm, workspace, ws_bytes, as_stream(stream));
}

// After the hash build the step reuses its scratch: [0, 256) the count of
// XPBD-labelled particles, then one bit per hash cell, then two float4 contact
// records per point.  A smaller workspace drops the records (and then the bits).
static size_t xpbd_bits_bytes(const int32_t *dims)
{
    const int64_t ncell = (int64_t)dims[0] * dims[1] * dims[2];
    return (size_t)((ncell + 31) / 32) * sizeof(unsigned);
}
static size_t xpbd_records_offset(const int32_t *dims) { return (256 + xpbd_bits_bytes(dims) + 255) / 256 * 256; }

// Workspace of the persistent step: a header (arrival counter, XPBD count, tile tickets,
// chunk sums of the in-kernel scan), the per-cell XPBD bits, then one area
// that holds the sort's buffers until the cell ranges are built and the
// contact records after that.
static size_t al256(size_t b) { return (b + 255) / 256 * 256; }
static size_t persist_area_offset(const int32_t *dims) { return al256(kPersistHeaderBytes + xpbd_bits_bytes(dims)); }
static size_t persist_sort_bytes(int64_t n)
{
    const int64_t hist_n = (int64_t)kRadix * sort_tiles(n);
    return al256(4 * (size_t)n) * 3 + al256(4 * (size_t)hist_n) * 2;
}
static size_t persist_workspace_bytes(int64_t n, const int32_t *dims)
{
    const size_t sort = persist_sort_bytes(n), rec = 2 * (size_t)n * sizeof(float4);
    return persist_area_offset(dims) + (sort > rec ? sort : rec);
}

size_t mpmw_xpbd_step_workspace_bytes(int64_t n, const int32_t *dims)
{
    if (n < 0) n = 0;
    const size_t hash = mpmw::hash_workspace_bytes(n);
    if (!dims) return hash;
    const size_t step = xpbd_records_offset(dims) + 2 * (size_t)n * sizeof(float4);
    const size_t pers = persist_workspace_bytes(n, dims);
    const size_t m = hash > step ? hash : step;
    return m > pers ? m : pers;
}

int mpmw_hash_build(const float *x, int64_t n, const mpmw_hash_t *h, void *workspace, size_t ws_bytes,
                    mpmw_stream_t stream)
{
    if (count_too_large(n, "hash_build")) return MPMW_E_ARG;
    TRY(check_hash(h, n));
    if (n < 0 || (n > 0 && (!x || !workspace))) { set_error("hash_build: bad arguments"); return MPMW_E_ARG; }
    return mpmw::hash_build(x, n, *h, workspace, ws_bytes, as_stream(stream));
}

int mpmw_xpbd_kernel(int which, const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                     const mpmw_xpbd_params_t *q, int flag, mpmw_stream_t stream)
{
    TRY(check_xpbd_args(p, x, q));
    if (p->n == 0) return MPMW_OK;
    cudaStream_t s = as_stream(stream);
    unsigned g = grid_for(p->n);
    switch (which) {
    case MPMW_XK_INTEGRATE: k_xpbd_integrate<<<g, kBlock, 0, s>>>(*p, *x, *q, flag); break;
    case MPMW_XK_RESET_LABELS: k_reset_labels<<<g, kBlock, 0, s>>>(*p); break;
    case MPMW_XK_BOUND: k_bound_contacts<<<g, kBlock, 0, s>>>(*p, *x, *q, flag); break;
    case MPMW_XK_PARTICLE:
        TRY(check_hash(h, p->n));
        k_particle_contacts<false><<<g, kBlock, 0, s>>>(*p, *x, *h, *q);
        break;
    case MPMW_XK_APPLY: k_apply_deltas<<<g, kBlock, 0, s>>>(*p, *x, *q, flag); break;
    case MPMW_XK_SLEEP:
        if (x->counts && flag && cudaMemsetAsync(x->counts, 0, 2 * sizeof(int), s) != cudaSuccess) {
            set_error("sleep: memset failed"); return MPMW_E_DEVICE;
        }
        if (!x->cum_dist) { set_error("sleep: cum_dist is required"); return MPMW_E_ARG; }
        k_sleep<<<g, kBlock, 0, s>>>(*p, *x, *q);
        break;
    case MPMW_XK_IMPULSES: k_impulses_commit<<<g, kBlock, 0, s>>>(*p, *x, *q, flag); break;
    case MPMW_XK_SWELL:
        if (!x->base_radius || !x->max_radius || !p->x_pc) { set_error("swell: radii and x_pc are required"); return MPMW_E_ARG; }
        k_swell<<<g, kBlock, 0, s>>>(*p, *x, *q);
        break;
    default: set_error("xpbd_kernel: unknown kernel %d", which); return MPMW_E_ARG;
    }
    return check_launch("xpbd kernel");
}

// process-wide choice of the step's form (1: one persistent launch where the
// workspace and the device allow it; 0: one launch per pass)
static std::atomic<int> g_xpbd_persistent{1};
static std::atomic<int64_t> g_xpbd_persistent_launches{0};

int64_t mpmw_xpbd_persistent_launches(void) { return g_xpbd_persistent_launches.load(); }

int mpmw_xpbd_set_options(int persistent)
{
    g_xpbd_persistent.store(persistent ? 1 : 0);
    return MPMW_OK;
}

// CTAs of the persistent step's cooperative grid on the current device (0: the
// device cannot launch it)
static int persist_grid_capacity()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 0;
    if (dev < 64) {
        const int c = cache[dev].load();
        if (c != 0) return c > 0 ? c : 0;
    }
    int coop = 0, sms = 0, per_sm = 0;
    int cap = -1;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_xpbd_step_persistent, kPersistThreads, 0) ==
            cudaSuccess &&
        per_sm > 0) {
        cap = per_sm * sms;
        if (cap > kPersistMaxCtas) cap = kPersistMaxCtas;
    }
    cudaGetLastError();
    if (dev < 64) cache[dev].store(cap);
    return cap > 0 ? cap : 0;
}

// The whole step as one cooperative launch of k_xpbd_step_persistent.
static int xpbd_step_persistent(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                                const mpmw_xpbd_params_t *q, uint32_t *status, void *workspace, int grid,
                                cudaStream_t s)
{
    const int64_t n = p->n;
    if (!x->cum_dist) { set_error("sleep: cum_dist is required"); return MPMW_E_ARG; }
    if (q->swelling_ratio > 0.f && (!x->base_radius || !x->max_radius || !p->x_pc)) {
        set_error("swell: radii and x_pc are required");
        return MPMW_E_ARG;
    }
    PersistArgs A;
    memset(&A, 0, sizeof(A));
    A.P = *p;
    A.X = *x;
    A.H = *h;
    A.q = *q;
    A.qi = *q;
    if (q->xpbd_only) A.qi.lock = 0;
    A.reset_labels = q->lock && !q->xpbd_only;
    A.hd = HashDims{{h->dims[0], h->dims[1], h->dims[2]}};
    A.inv = 1.0f / h->cell_width;
    A.ncell = (int64_t)h->dims[0] * h->dims[1] * h->dims[2];
    A.bit_words = (A.ncell + 31) / 32;
    int bits = 0;
    for (int64_t c = A.ncell - 1; c > 0; c >>= 1) ++bits;
    A.passes = (bits + kRadixBits - 1) / kRadixBits;
    A.ntiles = (int)sort_tiles(n);
    A.hist_n = (int64_t)kRadix * A.ntiles;
    char *w = static_cast<char *>(workspace);
    A.arrive = reinterpret_cast<unsigned *>(w);
    A.xpbd_count = reinterpret_cast<int *>(w) + 1;
    A.tickets = reinterpret_cast<unsigned *>(w) + 2;
    A.chunk_sums = reinterpret_cast<int *>(w) + 64;
    A.xpbd_cells = reinterpret_cast<unsigned *>(w + kPersistHeaderBytes);
    char *area = w + persist_area_offset(h->dims);
    A.keys_a = reinterpret_cast<int *>(area);
    A.keys_b = reinterpret_cast<int *>(area + al256(4 * (size_t)n));
    A.ids_scratch = reinterpret_cast<int *>(area + 2 * al256(4 * (size_t)n));
    A.hist = reinterpret_cast<int *>(area + 3 * al256(4 * (size_t)n));
    A.offs = reinterpret_cast<int *>(area + 3 * al256(4 * (size_t)n) + al256(4 * (size_t)A.hist_n));
    A.recA = reinterpret_cast<float4 *>(area);
    A.recB = A.recA + n;
    A.status = status;
    if (cudaMemsetAsync(w, 0, 3 * sizeof(int), s) != cudaSuccess ||
        (x->counts && cudaMemsetAsync(x->counts, 0, 2 * sizeof(int), s) != cudaSuccess)) {
        set_error("xpbd_step: memset failed");
        return MPMW_E_DEVICE;
    }
    void *args[] = {&A};
    if (cudaLaunchCooperativeKernel((const void *)k_xpbd_step_persistent, dim3((unsigned)grid), dim3(kPersistThreads),
                                    args, 0, s) != cudaSuccess) {
        set_error("xpbd_step: cooperative launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        return MPMW_E_DEVICE;
    }
    g_xpbd_persistent_launches.fetch_add(1);
    return MPMW_OK;
}

int mpmw_xpbd_step(const mpmw_particles_t *p, const mpmw_xpbd_t *x, const mpmw_hash_t *h,
                   const mpmw_xpbd_params_t *q, uint32_t *status, void *workspace, size_t ws_bytes,
                   mpmw_stream_t stream)
{
    TRY(check_xpbd_args(p, x, q));
    TRY(check_hash(h, p->n));
    if (p->n == 0) return MPMW_OK;
    cudaStream_t s = as_stream(stream);
    if (g_xpbd_persistent.load() && workspace && ws_bytes >= persist_workspace_bytes(p->n, h->dims) &&
        (reinterpret_cast<uintptr_t>(workspace) & 255u) == 0) {
        const int cap = persist_grid_capacity();
        if (cap > 0) {
            const int64_t work = (p->n + kPersistThreads - 1) / kPersistThreads;
            const int grid = (int)(work < cap ? (work > 0 ? work : 1) : cap);
            return xpbd_step_persistent(p, x, h, q, status, workspace, grid, s);
        }
    }
    TRY(mpmw_hash_build(p->x, p->n, h, workspace, ws_bytes, stream));
    // The hash build's scratch is free again: its first int counts the
    // particles labelled XPBD, which lets the contact passes skip a step
    // without any.
    int *xpbd_count = static_cast<int *>(workspace);
    if (cudaMemsetAsync(xpbd_count, 0, sizeof(int), s) != cudaSuccess) { set_error("xpbd_step: memset failed"); return MPMW_E_DEVICE; }
    // and, when it has room, one bit per hash cell holding an XPBD-labelled
    // particle, so that particles with none near them skip the neighbour walk
    unsigned *xpbd_cells = nullptr;
    {
        const int64_t ncell = (int64_t)h->dims[0] * h->dims[1] * h->dims[2];
        const size_t bits_bytes = (size_t)((ncell + 31) / 32) * sizeof(unsigned);
        if (ws_bytes >= 256 + bits_bytes) {
            xpbd_cells = reinterpret_cast<unsigned *>(static_cast<char *>(workspace) + 256);
            if (cudaMemsetAsync(xpbd_cells, 0, bits_bytes, s) != cudaSuccess) { set_error("xpbd_step: memset failed"); return MPMW_E_DEVICE; }
            HashDims hd{{h->dims[0], h->dims[1], h->dims[2]}};
            k_mark_xpbd_cells<<<grid_for(p->n), kBlock, 0, s>>>(*p, 1.0f / h->cell_width, hd, xpbd_cells);
            TRY(check_launch("k_mark_xpbd_cells"));
        }
    }
    float4 *recA = nullptr, *recB = nullptr;
    if (xpbd_cells && ws_bytes >= xpbd_records_offset(h->dims) + 2 * (size_t)p->n * sizeof(float4)) {
        recA = reinterpret_cast<float4 *>(static_cast<char *>(workspace) + xpbd_records_offset(h->dims));
        recB = recA + p->n;
    }
    // x_int <- x, v_int <- v for every particle (simulationRoutines.py:314-315), then integrate
    k_xpbd_integrate<<<grid_for(p->n), kBlock, 0, s>>>(*p, *x, *q, 3, xpbd_count);
    TRY(check_launch("k_xpbd_integrate"));
    if (q->lock && !q->xpbd_only) TRY(mpmw_xpbd_kernel(MPMW_XK_RESET_LABELS, p, x, h, q, 0, stream));
    mpmw_xpbd_params_t qi = *q;
    if (q->xpbd_only) qi.lock = 0;
    for (int it = 0; it < q->iterations; ++it) {
        TRY(mpmw_xpbd_kernel(MPMW_XK_BOUND, p, x, h, &qi, 0, stream));
        if (recA) {
            k_contact_records<<<grid_for(p->n), kBlock, 0, s>>>(*p, *x, *h, recA, recB, xpbd_count);
            TRY(check_launch("k_contact_records"));
            k_particle_contacts<true><<<grid_for(p->n), kBlock, 0, s>>>(*p, *x, *h, qi, xpbd_count, xpbd_cells,
                                                                       recA, recB);
        } else {
            k_particle_contacts<false><<<grid_for(p->n), kBlock, 0, s>>>(*p, *x, *h, qi, xpbd_count, xpbd_cells);
        }
        TRY(check_launch("k_particle_contacts"));
        TRY(mpmw_xpbd_kernel(MPMW_XK_APPLY, p, x, h, &qi, it == q->iterations - 1, stream));
    }
    TRY(mpmw_xpbd_kernel(MPMW_XK_SLEEP, p, x, h, q, 1, stream));
    TRY(mpmw_xpbd_kernel(MPMW_XK_IMPULSES, p, x, h, q, 1, stream));
    if (q->swelling_ratio > 0.f) TRY(mpmw_xpbd_kernel(MPMW_XK_SWELL, p, x, h, q, 0, stream));
    (void)s;
    return MPMW_OK;
}

}  // extern "C"
