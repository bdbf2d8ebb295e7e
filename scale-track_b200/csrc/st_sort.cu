/*
 * st_sort.cu -- periodic Morton re-sort of a cloud's parcels by owning cell, and the
 * kernels that hand the state back in the caller's order.
 *
 * Sorting keeps parcels of the same cell next to each other, so the warp-level run
 * reduction of the deposit collapses most of a tile into a few atomics, and neighbouring
 * warps gather neighbouring cells of U (L2 locality).  Keys are the Morton code of the cell
 * (i, j, k) (the linear cell index for meshes wider than 1024 cells, the owning tet on tet
 * meshes).  A key range wider than 2^24 values is coarsened to 2^24 by dropping low bits
 * (of each of i, j, k for Morton keys, of the index otherwise): neighbouring cells then share
 * a key, which keeps the locality the sort is for.  Keys are ranked by a counting sort: per-key
 * counts with one atomic per run of equal keys in a warp, an exclusive scan of the counts (two
 * kernels of this file), then each run claims its slots with one atomic.  Parcels of one run
 * keep their order; across runs and warps the order follows the order of the atomics, which no
 * result depends on (the deposit is an exact integer sum and everything else is per parcel).
 * Then every SoA array and the parcel id are gathered out of place into the other buffer.
 * The reference has no re-sort: its parcels keep their Hilbert ordered initial positions
 * inside each chunk (A:559-638).
 */
#include <cstdint>
#include <cuda_runtime.h>

#include "st_internal.h"

namespace st {

__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ float fl(float v) { return floorf(v); }
__device__ __forceinline__ double fl(double v) { return floor(v); }

/* cell (i,j,k) of a parcel clamped to the mesh; only an ordering key, never an index */
template <class P>
__device__ __forceinline__ void cell_ijk(const MeshK<P>& m, P x, P y, P z, int32_t& i,
                                         int32_t& j, int32_t& k)
{
    P fx = fl((x - m.origin[0]) * m.rD[0]);
    P fy = fl((y - m.origin[1]) * m.rD[1]);
    P fz = fl((z - m.origin[2]) * m.rD[2]);
    i = fx < (P)0 ? 0 : (fx >= (P)m.N[0] ? m.N[0] - 1 : (int32_t)fx);
    j = fy < (P)0 ? 0 : (fy >= (P)m.N[1] ? m.N[1] - 1 : (int32_t)fy);
    k = fz < (P)0 ? 0 : (fz >= (P)m.N[2] ? m.N[2] - 1 : (int32_t)fz);
}

/* shift: low bits dropped (of each of i, j, k for Morton keys, of the index otherwise) */
template <class P>
__global__ void k_sort_keys(const P* __restrict__ x, const P* __restrict__ y,
                            const P* __restrict__ z, int64_t n, MeshK<P> m, int morton,
                            int shift, uint32_t* __restrict__ keys)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        int32_t i, j, k;
        cell_ijk(m, x[p], y[p], z[p], i, j, k);
        const uint32_t key =
            morton ? (spread3((uint32_t)i >> shift) | (spread3((uint32_t)j >> shift) << 1) |
                      (spread3((uint32_t)k >> shift) << 2))
                   : ((uint32_t)(k * m.NxNy + j * m.N[0] + i) >> shift);
        keys[p] = key;
    }
}

/* Permutes the SoA arrays into sorted order.  Each thread handles GATHER_ILP outputs and
 * issues all their (scattered) loads before any store, so that many reads are in flight. */
constexpr int GATHER_ILP = 2;

/* tet meshes: the key is the owning tet (tets are numbered with spatial locality), less
 * `shift` low bits */
__global__ void k_sort_keys_cell(const int32_t* __restrict__ cell, int64_t n, int shift,
                                 uint32_t* __restrict__ keys)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        keys[p] = (uint32_t)cell[p] >> shift;
}

/* out[id[p]] = cell[p] */
__global__ void k_cells_unpermute(const int32_t* __restrict__ id, const int32_t* __restrict__ cell,
                                  int64_t n, int32_t* __restrict__ out)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        out[id[p]] = cell[p];
}

template <class P, class V>
__global__ void __launch_bounds__(256) k_gather(const uint32_t* __restrict__ perm, int64_t n,
                         const P* __restrict__ x0, const P* __restrict__ y0,
                         const P* __restrict__ z0, const V* __restrict__ u0,
                         const V* __restrict__ v0, const V* __restrict__ w0,
                         const V* __restrict__ d0, const int32_t* __restrict__ id0,
                         P* __restrict__ x1, P* __restrict__ y1, P* __restrict__ z1,
                         V* __restrict__ u1, V* __restrict__ v1, V* __restrict__ w1,
                         V* __restrict__ d1, int32_t* __restrict__ id1,
                         const int32_t* __restrict__ c0, int32_t* __restrict__ c1)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * GATHER_ILP;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x * GATHER_ILP + threadIdx.x; base < n;
         base += stride) {
        int64_t src[GATHER_ILP];
        P x[GATHER_ILP], y[GATHER_ILP], z[GATHER_ILP];
        V u[GATHER_ILP], v[GATHER_ILP], w[GATHER_ILP], dd[GATHER_ILP];
        int32_t id[GATHER_ILP];
        int32_t cc[GATHER_ILP];
#pragma unroll
        for (int k = 0; k < GATHER_ILP; ++k) {
            const int64_t p = base + (int64_t)k * blockDim.x;
            src[k] = p < n ? (int64_t)__ldcs(perm + p) : -1;
        }
#pragma unroll
        for (int k = 0; k < GATHER_ILP; ++k) {
            if (src[k] >= 0) {
                const int64_t s = src[k];
                x[k] = __ldg(x0 + s);
                y[k] = __ldg(y0 + s);
                z[k] = __ldg(z0 + s);
                u[k] = __ldg(u0 + s);
                v[k] = __ldg(v0 + s);
                w[k] = __ldg(w0 + s);
                dd[k] = __ldg(d0 + s);
                id[k] = __ldg(id0 + s);
                if (c0) cc[k] = __ldg(c0 + s);
            }
        }
#pragma unroll
        for (int k = 0; k < GATHER_ILP; ++k) {
            const int64_t p = base + (int64_t)k * blockDim.x;
            if (src[k] >= 0) {
                __stcs(x1 + p, x[k]);
                __stcs(y1 + p, y[k]);
                __stcs(z1 + p, z[k]);
                __stcs(u1 + p, u[k]);
                __stcs(v1 + p, v[k]);
                __stcs(w1 + p, w[k]);
                __stcs(d1 + p, dd[k]);
                __stcs(id1 + p, id[k]);
                if (c1) __stcs(c1 + p, cc[k]);
            }
        }
    }
}

/* out[id[p]] = in[p]: back to the order of st_set_parcels */
template <class P, class V>
__global__ void k_unpermute(const int32_t* __restrict__ id, int64_t n,
                            const P* __restrict__ x0, const P* __restrict__ y0,
                            const P* __restrict__ z0, const V* __restrict__ u0,
                            const V* __restrict__ v0, const V* __restrict__ w0,
                            const V* __restrict__ d0, P* __restrict__ x1, P* __restrict__ y1,
                            P* __restrict__ z1, V* __restrict__ u1, V* __restrict__ v1,
                            V* __restrict__ w1, V* __restrict__ d1)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = id[p];
        x1[t] = x0[p];
        y1[t] = y0[p];
        z1[t] = z0[p];
        u1[t] = u0[p];
        v1[t] = v0[p];
        w1[t] = w0[p];
        d1[t] = d0[p];
    }
}

/* Owning cell with the step's own locate semantics (A:680-693), 0-based, or -1 when the
 * position is outside the mesh. */
template <class P>
__device__ __forceinline__ int32_t cell_of(const MeshK<P>& m, P x, P y, P z)
{
    P fv[3] = {fl((x - m.origin[0]) * m.rD[0]), fl((y - m.origin[1]) * m.rD[1]),
               fl((z - m.origin[2]) * m.rD[2])};
    int32_t g[3];
    for (int a = 0; a < 3; ++a) {
        if (!(fv[a] >= (P)-2147483648.0 && fv[a] < (P)2147483648.0)) return -1;
        g[a] = (int32_t)fv[a];
    }
    int32_t q[3], r[3];
    for (int a = 0; a < 3; ++a) {
        q[a] = g[a] / m.N[a];
        r[a] = g[a] - q[a] * m.N[a];
    }
    const int32_t part = abs(q[2]) + abs(q[1]) + abs(q[0]) + 1;
    if (part != 1) return -1;
    return abs(r[2]) * m.NxNy + abs(r[1]) * m.N[0] + abs(r[0]);
}

/* Owning cell of every parcel (cell_of), written at the parcel's st_set_parcels index; a
 * count of the parcels outside the mesh. */
template <class P>
__global__ void k_cells(const P* __restrict__ x, const P* __restrict__ y,
                        const P* __restrict__ z, const int32_t* __restrict__ id, int64_t n,
                        MeshK<P> m, int32_t* __restrict__ cells, unsigned long long* outside)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cell_of(m, x[p], y[p], z[p]);
        if (c < 0 && outside) atomicAdd(outside, 1ULL);
        cells[id ? id[p] : p] = c;
    }
}

/* inv[id[p]] = p: the device position of every parcel by its st_set_parcels index */
__global__ void k_inverse_ids(const int32_t* __restrict__ id, int64_t n, uint32_t* __restrict__ inv)
{
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x)
        inv[id[p]] = (uint32_t)p;
}

/* The parcels ids[0..m) (st_set_parcels indices): state in FP64, out = [6][m] (x, y, z, u,
 * v, w), and the owning cell (the tracked tet when `cell` is given, else cell_of). */
template <class P, class V>
__global__ void k_sample(const uint32_t* __restrict__ inv, const int32_t* __restrict__ ids,
                         int64_t m, const P* __restrict__ x, const P* __restrict__ y,
                         const P* __restrict__ z, const V* __restrict__ u,
                         const V* __restrict__ v, const V* __restrict__ w,
                         const int32_t* __restrict__ cell, MeshK<P> mesh,
                         double* __restrict__ out, int32_t* __restrict__ cells_out)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = inv[ids[j]];
        out[j] = (double)x[p];
        out[m + j] = (double)y[p];
        out[2 * m + j] = (double)z[p];
        out[3 * m + j] = (double)u[p];
        out[4 * m + j] = (double)v[p];
        out[5 * m + j] = (double)w[p];
        cells_out[j] = cell ? cell[p] : cell_of(mesh, x[p], y[p], z[p]);
    }
}

/* ------------------------------------------------------------------------------------ */
/* counting sort                                                                        */
/* ------------------------------------------------------------------------------------ */
constexpr unsigned FULL_WARP = 0xffffffffu;
constexpr uint32_t NO_KEY = 0xffffffffu;   /* lanes past the end (keys are below 2^24) */

/* Runs of equal keys among a warp's 32 consecutive parcels (the input is close to sorted
 * between re-sorts): `heads` has a bit for the first lane of every run, `start` is the first
 * lane of this lane's run and `len` its length (used by the run's first lane).  Equal keys in
 * separate runs count and claim separately, which gives the same counts and distinct slots. */
__device__ __forceinline__ void key_run(uint32_t key, int lane, int& start, int& len, bool& head)
{
    const uint32_t prev = __shfl_up_sync(FULL_WARP, key, 1);
    head = lane == 0 || prev != key;
    const unsigned heads = __ballot_sync(FULL_WARP, head);
    start = 31 - __clz(heads & (FULL_WARP >> (31 - lane)));
    const unsigned later = lane == 31 ? 0u : heads & (FULL_WARP << (lane + 1));
    len = (later ? __ffs(later) - 1 : 32) - lane;
}

/* bins[key] += number of parcels with that key; one atomic per run of equal keys */
__global__ void k_bin_count(const uint32_t* __restrict__ keys, int64_t n, uint32_t nbins,
                            uint32_t* __restrict__ bins)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 < n;
         w += nw) {
        const int64_t p = w * 32 + lane;
        /* keys are below nbins by construction; the clamp only guards the bins */
        const uint32_t key = p < n ? min(__ldcs(keys + p), nbins - 1u) : NO_KEY;
        int start, len;
        bool head;
        key_run(key, lane, start, len, head);
        if (key != NO_KEY && head) atomicAdd(bins + key, (uint32_t)len);
    }
}

/* perm[slot] = p, slot = the key's offset + the parcel's place in its run of equal keys;
 * each run reserves its slots with one atomic (offsets are the exclusive scan of the counts
 * and move forward as slots are taken). */
__global__ void k_bin_rank(const uint32_t* __restrict__ keys, int64_t n, uint32_t nbins,
                           uint32_t* __restrict__ offsets, uint32_t* __restrict__ perm)
{
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w * 32 < n;
         w += nw) {
        const int64_t p = w * 32 + lane;
        const uint32_t key = p < n ? min(__ldcs(keys + p), nbins - 1u) : NO_KEY;
        int start, len;
        bool head;
        key_run(key, lane, start, len, head);
        uint32_t base = 0;
        if (key != NO_KEY && head) base = atomicAdd(offsets + key, (uint32_t)len);
        base = __shfl_sync(FULL_WARP, base, start);
        if (key != NO_KEY) perm[base + (uint32_t)(lane - start)] = (uint32_t)p;
    }
}

/* Exclusive scan of the per-key counts (up to 2^24 of them): k_scan_reduce sums a contiguous
 * chunk of the counts per block; k_scan_apply starts each block from the sum of the chunks
 * before it and scans its chunk in tiles of SCAN_TILE counts (four per thread, a warp
 * shuffle scan, then one over the warps' totals). */
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_TILE = 4 * SCAN_THREADS;
constexpr int SCAN_BLOCKS = 2 * 148;

/* sum of v over the block, returned to every thread */
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* wsum)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_WARP, v, o);
    if (lane == 0) wsum[warp] = v;
    __syncthreads();
    uint32_t t = lane < nw ? wsum[lane] : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL_WARP, t, o);
    __syncthreads();
    return t;
}

/* exclusive prefix of v over the block's threads; `total` = the block's sum */
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* wsum, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL_WARP, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL_WARP, w, o);
            if (lane >= o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    const uint32_t before = warp ? wsum[warp - 1] : 0u;
    total = wsum[nw - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t* __restrict__ in,
                                                              int64_t n, int64_t chunk,
                                                              uint32_t* __restrict__ partials)
{
    __shared__ uint32_t wsum[32];
    const int64_t begin = blockIdx.x * chunk;
    const int64_t end = begin + chunk < n ? begin + chunk : n;
    uint32_t v = 0;
    for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) v += __ldcs(in + i);
    v = block_sum(v, wsum);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const uint32_t* __restrict__ in,
                                                             int64_t n, int64_t chunk,
                                                             const uint32_t* __restrict__ partials,
                                                             uint32_t* __restrict__ out)
{
    __shared__ uint32_t wsum[32];
    uint32_t c = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += blockDim.x) c += partials[j];
    uint32_t carry = block_sum(c, wsum);
    const int64_t begin = blockIdx.x * chunk;
    const int64_t end = begin + chunk < n ? begin + chunk : n;
    for (int64_t t0 = begin; t0 < end; t0 += SCAN_TILE) {
        const int64_t idx = t0 + 4 * (int64_t)threadIdx.x;
        uint32_t v[4] = {0u, 0u, 0u, 0u};
        if (idx + 4 <= end) {
            const uint4 q = *reinterpret_cast<const uint4*>(in + idx);
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else {
            for (int e = 0; e < 4; ++e)
                if (idx + e < end) v[e] = in[idx + e];
        }
        uint32_t total;
        uint32_t run = carry + block_exclusive((v[0] + v[1]) + (v[2] + v[3]), wsum, total);
        uint32_t o[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            o[e] = run;
            run += v[e];
        }
        if (idx + 4 <= end) {
            *reinterpret_cast<uint4*>(out + idx) = make_uint4(o[0], o[1], o[2], o[3]);
        } else {
            for (int e = 0; e < 4; ++e)
                if (idx + e < end) out[idx + e] = o[e];
        }
        carry += total;
    }
}

/* out = exclusive scan of in[0..n); partials holds SCAN_BLOCKS counts */
static cudaError_t scan_counts(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* partials,
                               cudaStream_t s)
{
    int64_t chunk = (n + SCAN_BLOCKS - 1) / SCAN_BLOCKS;
    chunk = (chunk + 3) / 4 * 4;   /* chunks start on 16-byte boundaries */
    k_scan_reduce<<<SCAN_BLOCKS, SCAN_THREADS, 0, s>>>(in, n, chunk, partials);
    k_scan_apply<<<SCAN_BLOCKS, SCAN_THREADS, 0, s>>>(in, n, chunk, partials, out);
    return cudaGetLastError();
}

size_t count_sort_scan_bytes(int key_bits)
{
    (void)key_bits;
    return SCAN_BLOCKS * sizeof(uint32_t);
}

static int grid_for(int64_t n)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    return (int)g;
}

template <class P, class V>
cudaError_t sort_cloud(SortBufs<P, V>& b, int cur, int64_t n, const MeshK<P>& mesh, int key_bits,
                       int key_shift, bool morton, cudaStream_t s, int* launches)
{
    if (n <= 1) return cudaSuccess;
    if (!b.bins || key_bits > COUNT_SORT_MAX_BITS) return cudaErrorInvalidValue;
    const int o = 1 - cur;
    if (b.cell[cur])
        k_sort_keys_cell<<<grid_for(n), 256, 0, s>>>(b.cell[cur], n, key_shift, b.keys[0]);
    else
        k_sort_keys<P><<<grid_for(n), 256, 0, s>>>(b.x[cur], b.y[cur], b.z[cur], n, mesh,
                                                   morton ? 1 : 0, key_shift, b.keys[0]);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int64_t nbins = (int64_t)1 << key_bits;
    if ((e = cudaMemsetAsync(b.bins, 0, nbins * sizeof(uint32_t), s)) != cudaSuccess) return e;
    const int wg = grid_for(n);
    k_bin_count<<<wg, 256, 0, s>>>(b.keys[0], n, (uint32_t)nbins, b.bins);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = scan_counts(b.bins, b.offsets, nbins, static_cast<uint32_t*>(b.scan_temp), s)) !=
        cudaSuccess)
        return e;
    k_bin_rank<<<wg, 256, 0, s>>>(b.keys[0], n, (uint32_t)nbins, b.offsets, b.perm[1]);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    int64_t gblocks = (n + 256 * GATHER_ILP - 1) / (256 * GATHER_ILP);
    if (gblocks > 148 * 64) gblocks = 148 * 64;
    k_gather<P, V><<<(int)gblocks, 256, 0, s>>>(b.perm[1], n, b.x[cur], b.y[cur], b.z[cur],
                                               b.u[cur], b.v[cur], b.w[cur], b.d[cur],
                                               b.id[cur], b.x[o], b.y[o], b.z[o], b.u[o],
                                               b.v[o], b.w[o], b.d[o], b.id[o], b.cell[cur],
                                               b.cell[o]);
    /* keys, counts, the two scan kernels, slots, gather */
    if (launches) *launches += 6;
    return cudaGetLastError();
}

template <class P, class V>
cudaError_t unpermute_cloud(SortBufs<P, V>& b, int cur, int64_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    const int o = 1 - cur;
    k_unpermute<P, V><<<grid_for(n), 256, 0, s>>>(b.id[cur], n, b.x[cur], b.y[cur], b.z[cur],
                                                  b.u[cur], b.v[cur], b.w[cur], b.d[cur],
                                                  b.x[o], b.y[o], b.z[o], b.u[o], b.v[o],
                                                  b.w[o], b.d[o]);
    return cudaGetLastError();
}

template <class P>
cudaError_t cells_cloud(const P* x, const P* y, const P* z, const int32_t* id, int64_t n,
                        const MeshK<P>& mesh, int32_t* cells_out, unsigned long long* outside,
                        cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_cells<P><<<grid_for(n), 256, 0, s>>>(x, y, z, id, n, mesh, cells_out, outside);
    return cudaGetLastError();
}

template <class P, class V>
cudaError_t sample_cloud(SortBufs<P, V>& b, int cur, int64_t n, const MeshK<P>& mesh,
                         const int32_t* ids, int64_t m, double* out, int32_t* cells_out,
                         cudaStream_t s)
{
    if (m == 0) return cudaSuccess;
    /* the sort's permutation buffer is free between steps: it holds the inverse of the ids */
    k_inverse_ids<<<grid_for(n), 256, 0, s>>>(b.id[cur], n, b.perm[0]);
    k_sample<P, V><<<grid_for(m), 256, 0, s>>>(b.perm[0], ids, m, b.x[cur], b.y[cur], b.z[cur],
                                               b.u[cur], b.v[cur], b.w[cur], b.cell[cur], mesh,
                                               out, cells_out);
    return cudaGetLastError();
}

cudaError_t cells_unpermute(const int32_t* id, const int32_t* cell, int64_t n, int32_t* out,
                            cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_cells_unpermute<<<grid_for(n), 256, 0, s>>>(id, cell, n, out);
    return cudaGetLastError();
}

#define ST_INST(P, V)                                                                         \
    template cudaError_t sort_cloud<P, V>(SortBufs<P, V>&, int, int64_t, const MeshK<P>&, int, \
                                          int, bool, cudaStream_t, int*);                     \
    template cudaError_t unpermute_cloud<P, V>(SortBufs<P, V>&, int, int64_t, cudaStream_t); \
    template cudaError_t sample_cloud<P, V>(SortBufs<P, V>&, int, int64_t, const MeshK<P>&,    \
                                            const int32_t*, int64_t, double*, int32_t*,        \
                                            cudaStream_t);
ST_INST(float, float)
ST_INST(double, float)
ST_INST(double, double)
template cudaError_t cells_cloud<float>(const float*, const float*, const float*,
                                        const int32_t*, int64_t, const MeshK<float>&, int32_t*,
                                        unsigned long long*, cudaStream_t);
template cudaError_t cells_cloud<double>(const double*, const double*, const double*,
                                         const int32_t*, int64_t, const MeshK<double>&, int32_t*,
                                         unsigned long long*, cudaStream_t);

}  // namespace st
