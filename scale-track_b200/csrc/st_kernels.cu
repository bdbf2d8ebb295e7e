/*
 * st_kernels.cu -- the parcel step and the source reduction, written for sm_100a.
 *
 * One warp owns a tile of 32 consecutive parcels; lanes read the SoA arrays with
 * consecutive addresses (streaming loads, issued one tile ahead, that do not displace the
 * L2-resident cell arrays), gather the cell velocity, run the substeps in registers and
 * write back.
 * The deposit of each parcel into its cell (A:1342-1345, A:1361) is reduced inside the warp
 * over runs of equal cells (parcels are kept Morton-sorted by cell, so neighbours mostly
 * share a cell) and only the last lane of each run touches memory.
 *
 * Deterministic deposit: every deposit component is scaled by 2^-L and rounded to a 64-bit
 * integer, so the per-cell sums are integer sums and do not depend on which warp adds
 * first.  L follows the largest deposit of the previous step (CloudCtl).  With one limb the
 * headroom covers any distribution of the cloud's deposits over cells; two limbs (FP64
 * mode) carry 32 more bits of resolution.  A finalize pass converts the integers to FP64
 * and clears the accumulators for the next step.
 *
 * Reference: A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 *   evolve_on_device!  A:1258-1269     evolve_particle!  A:1271-1365
 *   locate             A:663-697       update! (GPU)     A:710-728
 * Compiled with --fmad=false: the reference's arithmetic has no fused multiply-adds.
 */
#include <cstdint>
#include <cuda_runtime.h>

#include "st_step.cuh"

namespace st {

/* ------------------------------------------------------------------------------------ */
/* the step kernel                                                                      */
/* ------------------------------------------------------------------------------------ */

constexpr int TILE = WARP_TILE;      /* parcels per warp tile (CloudK::tile0 counts these) */
constexpr int SLICES = TILE / 32;    /* 32-parcel slices per warp tile */

template <class P, class V>
__device__ __forceinline__ int find_cloud(const StepArgs<P, V>& a, int64_t tile)
{
    int lo = 0, hi = a.nclouds - 1;
    while (lo < hi) {  /* last cloud whose tile0 <= tile */
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&a.clouds[mid].tile0) <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/* The step kernel.  A warp owns a tile of SLICES x 32 consecutive parcels (lane l holds
 * parcels l, l+32, l+64, l+96 of the tile): all loads of the tile are issued one tile ahead
 * (while the previous tile is stepped), then the start cells are located and the cell
 * velocities gathered for every slice, then each slice is stepped, stored and its deposits
 * reduced.  Tiles are distributed over the persistent grid with a fixed stride; the clouds
 * of a multi-cloud launch occupy consecutive tile ranges. */
/* Resident blocks of 256 threads per SM the compiler must allow (a register budget):
 * 3 (80 registers), which holds the two tiles of the software pipeline without spills. */
#ifndef ST_MIN_BLOCKS
#define ST_MIN_BLOCKS 3
#endif
#ifndef ST_MIN_BLOCKS_FP64
#define ST_MIN_BLOCKS_FP64 3
#endif
/* Several substeps per call (the multi-cloud workload) keep more state live per parcel. */
#ifndef ST_MIN_BLOCKS_SUB
#define ST_MIN_BLOCKS_SUB 3
#endif
template <class V, bool ONE>
struct MinBlocks {
    static constexpr int value =
        sizeof(V) == 8 ? ST_MIN_BLOCKS_FP64 : (ONE ? ST_MIN_BLOCKS : ST_MIN_BLOCKS_SUB);
};

template <class P, class V, int DEP, bool ONE, bool SINGLE>
__global__ void __launch_bounds__(256, MinBlocks<V, ONE>::value) k_step(const StepArgs<P, V> a)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr bool DET = (DEP == DEP_DET1 || DEP == DEP_DET2);

    if (!ONE) {   /* the table of x^0.687 serves the multi-substep loop */
        pow_tab_fill();
        __syncthreads();
    }
    int cur = -1;
    Quant qp = {0.0, 0.0, 0};
    AmaxT<V> amax = (V)0;
    unsigned ovf = 0, nlost = 0;

    /* Software pipeline over the warp's tiles (one substep): the streaming loads of the next
     * tile are issued before the current tile is stepped, so each warp keeps two tiles of
     * parcel data in flight and the HBM latency overlaps the arithmetic.  With several
     * substeps the kernel is bound by their arithmetic, the loads are a small share of it,
     * and the second tile's registers would spill in the substep loop: each tile is loaded
     * when it is stepped. */
    constexpr bool AHEAD = ONE;
    struct Raw {
        P X[SLICES], Y[SLICES], Z[SLICES];
        V Uv[SLICES], Vv[SLICES], Wv[SLICES], D[SLICES];
    };
    auto load = [&](int64_t t, Raw& r) {   /* every load of tile t (streaming, evict-first) */
        const int cc = SINGLE ? 0 : find_cloud(a, t);
        const CloudK<P, V>& cl = SINGLE ? a.one : a.clouds[cc];
        const int64_t n = cl.n;
        const int64_t base = (t - cl.tile0) * TILE + lane;
#pragma unroll
        for (int s = 0; s < SLICES; ++s) {
            const int64_t i = base + 32 * s;
            if (i < n) {
                r.X[s] = ld_stream(cl.x + i);
                r.Y[s] = ld_stream(cl.y + i);
                r.Z[s] = ld_stream(cl.z + i);
                r.Uv[s] = ld_stream(cl.u + i);
                r.Vv[s] = ld_stream(cl.v + i);
                r.Wv[s] = ld_stream(cl.w + i);
                r.D[s] = ld_stream(cl.d + i);
            }
        }
    };
    Raw R, RN;
    if (AHEAD && warp0 < a.total_tiles) load(warp0, R);
    for (int64_t tile = warp0; tile < a.total_tiles; tile += nwarps) {
        if (!AHEAD)
            load(tile, R);
        else if (tile + nwarps < a.total_tiles)
            load(tile + nwarps, RN);
        const int c = SINGLE ? 0 : find_cloud(a, tile);
        if (c != cur) {
            if (cur >= 0) flush_ctl<DEP>(a.ctl + cur, lane, amax, ovf, nlost);
            cur = c;
            if (DET) qp = make_quant(a.ctl[c].L, a.ctl[c].H + QUANT_GROWTH_BITS);
        }
        const CloudK<P, V>& cl = SINGLE ? a.one : a.clouds[c];
        const int64_t n = cl.n;
        const int64_t base = (tile - cl.tile0) * TILE + lane;
        unsigned long long* const acc = DET ? cl.acc : nullptr;
        double* const src = (DEP == DEP_ATOMIC) ? cl.src : nullptr;
        P X[SLICES], Y[SLICES], Z[SLICES];
        V Uv[SLICES], Vv[SLICES], Wv[SLICES], D[SLICES];
#pragma unroll
        for (int s = 0; s < SLICES; ++s) {
            X[s] = R.X[s]; Y[s] = R.Y[s]; Z[s] = R.Z[s];
            Uv[s] = R.Uv[s]; Vv[s] = R.Vv[s]; Wv[s] = R.Wv[s]; D[s] = R.D[s];
        }
        if (AHEAD) R = RN;
        /* phase 2: start cells (A:1286) and raw cell velocities (A:1288; the fluid factor is
         * applied in the slip) */
        int32_t pI[SLICES];
        V Ur[SLICES][3];
#pragma unroll
        for (int s = 0; s < SLICES; ++s) {
            pI[s] = 0;
            if (base + 32 * s < n) {
                bool bad = false;
                LocK l0 = locate(a.mesh, X[s], Y[s], Z[s], bad);
                if (!bad && l0.part == 1) {
                    pI[s] = l0.posI;
                    const V* Uc = a.U + 3 * (int64_t)(l0.posI - 1);
                    Ur[s][0] = __ldg(Uc);
                    Ur[s][1] = __ldg(Uc + 1);
                    Ur[s][2] = __ldg(Uc + 2);
                } else {
                    ++nlost;
                }
            }
        }
        /* phase 3: substeps, store, deposit, one slice after the other */
#pragma unroll
        for (int s = 0; s < SLICES; ++s) {
            const int64_t i = base + 32 * s;
            int32_t key = -1;
            V dep[3] = {(V)0, (V)0, (V)0};
            if (pI[s] > 0) {
                P pos[3] = {X[s], Y[s], Z[s]};
                V vel[3] = {Uv[s], Vv[s], Wv[s]};
                bool lost = false;
                if (ONE) {
                    evolve_one<P, V>(a, pos, vel, D[s] * a.phys.dscale, pI[s], Ur[s], lost, dep);
                    key = pI[s] - 1;
                } else {
                    evolve_parcel<P, V, DEP>(a, pos, vel, D[s] * a.phys.dscale, pI[s], Ur[s],
                                             acc, src, qp, amax, ovf, lost, key, dep);
                }
                if (lost) {
                    ++nlost;
                    key = -1;
                } else if (DEP != DEP_PROBE) {                                   /* A:1355-1360 */
                    /* the array pointers are read here, after the substeps, not held in
                     * registers through them */
                    st_stream(cl.x + i, pos[0]);
                    st_stream(cl.y + i, pos[1]);
                    st_stream(cl.z + i, pos[2]);
                    st_stream(cl.u + i, vel[0]);
                    st_stream(cl.v + i, vel[1]);
                    st_stream(cl.w + i, vel[2]);
                }
            }
            deposit_warp<DEP, V>(key, dep, acc, src, qp, lane, amax, ovf);
        }
    }
    if (cur >= 0) flush_ctl<DEP>(a.ctl + cur, lane, amax, ovf, nlost);
}

template <class P, class V, bool ONE, bool SINGLE>
static cudaError_t launch_step_t(const StepArgs<P, V>& a, int dep, int grid, int block,
                                 cudaStream_t s)
{
    switch (dep) {
    case DEP_DET1: k_step<P, V, DEP_DET1, ONE, SINGLE><<<grid, block, 0, s>>>(a); break;
    case DEP_DET2: k_step<P, V, DEP_DET2, ONE, SINGLE><<<grid, block, 0, s>>>(a); break;
    case DEP_ATOMIC: k_step<P, V, DEP_ATOMIC, ONE, SINGLE><<<grid, block, 0, s>>>(a); break;
    case DEP_PROBE: k_step<P, V, DEP_PROBE, ONE, SINGLE><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class P, class V>
cudaError_t launch_step(const StepArgs<P, V>& a, int dep, int grid, int block, cudaStream_t s)
{
    if (a.nclouds == 1)
        return a.phys.nsub == 1 ? launch_step_t<P, V, true, true>(a, dep, grid, block, s)
                                : launch_step_t<P, V, false, true>(a, dep, grid, block, s);
    return a.phys.nsub == 1 ? launch_step_t<P, V, true, false>(a, dep, grid, block, s)
                            : launch_step_t<P, V, false, false>(a, dep, grid, block, s);
}

template <class P, class V, bool ONE, bool SINGLE>
static int max_active_t(int dep, int block)
{
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (dep) {
    case DEP_DET1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_DET1, ONE, SINGLE>, block, 0); break;
    case DEP_DET2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_DET2, ONE, SINGLE>, block, 0); break;
    case DEP_ATOMIC: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_ATOMIC, ONE, SINGLE>, block, 0); break;
    case DEP_PROBE: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_PROBE, ONE, SINGLE>, block, 0); break;
    default: break;
    }
    return e == cudaSuccess ? nb : 0;
}

template <class P, class V>
int step_max_active_blocks(int dep, int block)
{
    /* all variants are compiled with the same launch bounds; take the smallest */
    int m = max_active_t<P, V, true, true>(dep, block);
    const int r[3] = {max_active_t<P, V, false, true>(dep, block),
                      max_active_t<P, V, true, false>(dep, block),
                      max_active_t<P, V, false, false>(dep, block)};
    for (int v : r) m = v < m ? v : m;
    return m;
}

template cudaError_t launch_step<float, float>(const StepArgs<float, float>&, int, int, int, cudaStream_t);
template cudaError_t launch_step<double, float>(const StepArgs<double, float>&, int, int, int, cudaStream_t);
template cudaError_t launch_step<double, double>(const StepArgs<double, double>&, int, int, int, cudaStream_t);
template int step_max_active_blocks<float, float>(int, int);
template int step_max_active_blocks<double, float>(int, int);
template int step_max_active_blocks<double, double>(int, int);

/* ------------------------------------------------------------------------------------ */
/* source finalize: fixed point -> FP64, clear accumulators, next scale                 */
/* ------------------------------------------------------------------------------------ */

template <int LIMBS>
__global__ void __launch_bounds__(256) k_finalize(unsigned long long* __restrict__ acc,
                                                  double* __restrict__ src,
                                                  float* __restrict__ src32, CloudCtl* ctl,
                                                  const int32_t* __restrict__ Lsrc,
                                                  unsigned int* counter, int nclouds,
                                                  int64_t stride)
{
    /* stride: per-cloud component count, a multiple of 4 (padding stays zero).  The caller
     * clears the accumulators after this kernel.  Lsrc: the scale of each cloud when the next
     * scale was already set by k_next_scale (overlapped finalize), else null. */
    const int c = blockIdx.y;
    const int L = Lsrc ? Lsrc[c] : ctl[c].L;
    const ulonglong2* a = reinterpret_cast<const ulonglong2*>(acc + (int64_t)c * stride * LIMBS);
    double2* s = reinterpret_cast<double2*>(src + (int64_t)c * stride);
    float4* s32 = src32 ? reinterpret_cast<float4*>(src32 + (int64_t)c * stride) : nullptr;
    const int64_t ngroups = stride / 4;
    const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
    /* read-only pass: the accumulators are cleared afterwards by a memset, which costs less
     * than writing zeros back into the lines just read; the source is streamed out */
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gstride) {
        double v[4];
        if (LIMBS == 1) {
            ulonglong2 q0 = __ldcs(a + 2 * g);
            ulonglong2 q1 = __ldcs(a + 2 * g + 1);
            v[0] = (double)(long long)q0.x;
            v[1] = (double)(long long)q0.y;
            v[2] = (double)(long long)q1.x;
            v[3] = (double)(long long)q1.y;
        } else {
            ulonglong2 q[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) q[k] = __ldcs(a + 4 * g + k);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                long long hi = (long long)q[k].x;
                unsigned long long lo = q[k].y;
                hi += (long long)(lo >> 32);
                lo &= 0xffffffffULL;
                v[k] = (double)hi * 4294967296.0 + (double)lo;
            }
        }
        const double o[4] = {ldexp2(v[0], L), ldexp2(v[1], L), ldexp2(v[2], L),
                             ldexp2(v[3], L)};
        __stcs(s + 2 * g, make_double2(o[0], o[1]));
        __stcs(s + 2 * g + 1, make_double2(o[2], o[3]));
        /* a 4-byte copy for an FP32 exchange array, rounded once from the FP64 source */
        if (s32) __stcs(s32 + g, make_float4((float)o[0], (float)o[1], (float)o[2], (float)o[3]));
    }
    /* the last block to finish moves every cloud to the scale of its largest deposit */
    if (Lsrc) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int ticket = atomicAdd(counter, 1u);
        if (ticket == gridDim.x * gridDim.y - 1) {
            __threadfence();
            for (int k = 0; k < nclouds; ++k) {
                volatile CloudCtl* q = ctl + k;
                int em = q->emax;
                if (em != EXP_NONE) q->L = em - q->H;
                q->emax = EXP_NONE;
            }
            *counter = 0u;
            __threadfence();
        }
    }
}

cudaError_t launch_finalize(int limbs, unsigned long long* acc, double* src, float* src32,
                            CloudCtl* ctl, const int32_t* Lsrc, unsigned int* counter,
                            int nclouds, int64_t stride, int grid_x, cudaStream_t s)
{
    if (stride % 4) return cudaErrorInvalidValue;
    dim3 grid(grid_x, nclouds);
    if (limbs == 1)
        k_finalize<1><<<grid, 256, 0, s>>>(acc, src, src32, ctl, Lsrc, counter, nclouds, stride);
    else
        k_finalize<2><<<grid, 256, 0, s>>>(acc, src, src32, ctl, Lsrc, counter, nclouds, stride);
    return cudaGetLastError();
}

/* The scale bookkeeping of k_finalize on its own, for an overlapped finalize: keeps each
 * cloud's scale of the step just run in Lfin (for the finalize on the other stream) and moves
 * the cloud to the scale of that step's largest deposit for the next step. */
__global__ void k_next_scale(CloudCtl* ctl, int32_t* Lfin, int nclouds)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nclouds) {
        Lfin[k] = ctl[k].L;
        const int em = ctl[k].emax;
        if (em != EXP_NONE) ctl[k].L = em - ctl[k].H;
        ctl[k].emax = EXP_NONE;
    }
}

cudaError_t launch_next_scale(CloudCtl* ctl, int32_t* Lfin, int nclouds, cudaStream_t s)
{
    k_next_scale<<<(nclouds + 127) / 128, 128, 0, s>>>(ctl, Lfin, nclouds);
    return cudaGetLastError();
}

/* After a probe pass: the scale of the first step maps the largest deposit to 2^H. */
__global__ void k_set_scale(CloudCtl* ctl, int nclouds)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nclouds) {
        int em = ctl[k].emax;
        ctl[k].L = (em == EXP_NONE) ? -ctl[k].H : em - ctl[k].H;
        ctl[k].emax = EXP_NONE;
    }
}

/* Copies every cloud's largest-deposit exponent between the control blocks and a contiguous
 * array (to_ctl: array -> blocks), the buffer a sharded run max-reduces across ranks. */
__global__ void k_ctl_exponents(CloudCtl* ctl, int32_t* e, int nclouds, int to_ctl)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nclouds) {
        if (to_ctl) ctl[k].emax = e[k];
        else e[k] = ctl[k].emax;
    }
}

cudaError_t launch_ctl_exponents(CloudCtl* ctl, int32_t* e, int nclouds, bool to_ctl,
                                 cudaStream_t s)
{
    k_ctl_exponents<<<(nclouds + 127) / 128, 128, 0, s>>>(ctl, e, nclouds, to_ctl ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_set_scale(CloudCtl* ctl, int nclouds, cudaStream_t s)
{
    k_set_scale<<<(nclouds + 127) / 128, 128, 0, s>>>(ctl, nclouds);
    return cudaGetLastError();
}

__global__ void k_zero_f64(double* p, int64_t n)
{
    /* n is a multiple of 2 and p 16-byte aligned (padded per-cloud strides) */
    double2* q = reinterpret_cast<double2*>(p);
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n / 2;
         j += (int64_t)gridDim.x * blockDim.x)
        q[j] = make_double2(0.0, 0.0);
}

cudaError_t launch_zero_f64(double* p, int64_t n, cudaStream_t s)
{
    int grid = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
    if (grid < 1) grid = 1;
    k_zero_f64<<<grid, 256, 0, s>>>(p, n);
    return cudaGetLastError();
}

__global__ void k_f64_to_f32(const double* __restrict__ in, float* __restrict__ out, int64_t n)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        out[j] = (float)in[j];
}

/* Element-wise conversion between FP32 and FP64 arrays; either side may be mapped host
 * memory (the zero-copy exchange reads U from and writes the source to it directly). */
template <class I, class O>
__global__ void k_convert(const I* __restrict__ in, O* __restrict__ out, int64_t n)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        out[j] = (O)in[j];
}

cudaError_t launch_convert(const void* in, int in_bytes, void* out, int out_bytes, int64_t n,
                           cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    if (in_bytes == 4 && out_bytes == 4)
        k_convert<float, float><<<(int)g, 256, 0, s>>>((const float*)in, (float*)out, n);
    else if (in_bytes == 4)
        k_convert<float, double><<<(int)g, 256, 0, s>>>((const float*)in, (double*)out, n);
    else if (out_bytes == 4)
        k_convert<double, float><<<(int)g, 256, 0, s>>>((const double*)in, (float*)out, n);
    else
        k_convert<double, double><<<(int)g, 256, 0, s>>>((const double*)in, (double*)out, n);
    return cudaGetLastError();
}

/* Constant extrapolation of the source (A:742-747): est = 2 S - est_prev, in place on
 * `est`, with S = 0 when there is no completed step yet (s == nullptr); the FP32 copy for a
 * 4-byte exchange array is written alongside. */
__global__ void k_extrapolate(const double* __restrict__ s, double* __restrict__ est,
                             float* __restrict__ est32, int64_t n)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        const double e = (s ? 2.0 * s[j] : 0.0) - est[j];
        est[j] = e;
        if (est32) est32[j] = (float)e;
    }
}

cudaError_t launch_extrapolate(const double* s, double* est, float* est32, int64_t n,
                               cudaStream_t st)
{
    int64_t g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    if (g < 1) g = 1;
    k_extrapolate<<<(int)g, 256, 0, st>>>(s, est, est32, n);
    return cudaGetLastError();
}

__global__ void k_f32_to_f64(const float* __restrict__ in, double* __restrict__ out, int64_t n)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        out[j] = (double)in[j];
}

cudaError_t launch_f64_to_f32(const double* in, float* out, int64_t n, cudaStream_t s)
{
    int grid = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
    if (grid < 1) grid = 1;
    k_f64_to_f32<<<grid, 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_f32_to_f64(const float* in, double* out, int64_t n, cudaStream_t s)
{
    int grid = (int)((n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8);
    if (grid < 1) grid = 1;
    k_f32_to_f64<<<grid, 256, 0, s>>>(in, out, n);
    return cudaGetLastError();
}

}  // namespace st
