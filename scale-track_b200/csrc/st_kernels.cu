/*
 * st_kernels.cu -- the parcel step and the source reduction, written for sm_100a.
 *
 * One warp owns a tile of 32 consecutive parcels; lanes read the SoA arrays with
 * consecutive addresses (streaming loads that do not displace the L2-resident cell arrays),
 * gather the cell velocity, run the substeps in registers and write back.  The deposit of
 * each parcel into its cell (A:1342-1345, A:1361) is reduced inside the warp over runs of
 * equal cells (parcels are kept Morton-sorted by cell, so neighbours mostly share a cell)
 * and only the last lane of each run touches memory.
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

#include "st_internal.h"
#include "st_pow.h"

namespace st {

#define FULL_MASK 0xffffffffu

/* ------------------------------------------------------------------------------------ */
/* relocation                                                                           */
/* ------------------------------------------------------------------------------------ */

__device__ __forceinline__ float st_floor(float v) { return floorf(v); }
__device__ __forceinline__ double st_floor(double v) { return floor(v); }
__device__ __forceinline__ float st_sqrt(float v) { return __fsqrt_rn(v); }
__device__ __forceinline__ double st_sqrt(double v) { return __dsqrt_rn(v); }

/* floor(label, v) (A:668-670); values outside int32 mark the parcel as lost. */
template <class P>
__device__ __forceinline__ int32_t floor_label(P v, bool& bad)
{
    P f = st_floor(v);
    if (!(f >= (P)-2147483648.0 && f < (P)2147483648.0)) {
        bad = true;
        return 0;
    }
    return (int32_t)f;
}

struct LocK {
    int32_t I, J, K;
    int32_t posI;   /* 1-based linear cell index */
    int32_t part;   /* 1-based partition index (one partition) */
};

/* divrem(i, n) truncating toward zero; most parcels are inside, where it is (0, i). */
__device__ __forceinline__ void divrem_label(int32_t i, int32_t n, int32_t& q, int32_t& r)
{
    if ((uint32_t)i < (uint32_t)n) {
        q = 0;
        r = i;
    } else {
        q = i / n;
        r = i - q * n;
    }
}

template <class P>
__device__ __forceinline__ LocK locate(const MeshK<P>& m, P x, P y, P z, bool& bad)
{
    LocK r;
    r.I = floor_label((x - m.origin[0]) * m.rD[0], bad);
    r.J = floor_label((y - m.origin[1]) * m.rD[1], bad);
    r.K = floor_label((z - m.origin[2]) * m.rD[2], bad);
    int32_t iP, iL, jP, jL, kP, kL;
    divrem_label(r.I, m.N[0], iP, iL);
    divrem_label(r.J, m.N[1], jP, jL);
    divrem_label(r.K, m.N[2], kP, kL);
    r.part = abs(kP) + abs(jP) + abs(iP) + 1;
    r.posI = abs(kL) * m.NxNy + abs(jL) * m.N[0] + abs(iL) + 1;
    return r;
}

/* ------------------------------------------------------------------------------------ */
/* fixed-point deposit                                                                  */
/* ------------------------------------------------------------------------------------ */

/* smallest e with |a| < 2^e, for finite a != 0 (the frexp exponent) */
__device__ __forceinline__ int exp_of(double a)
{
    uint64_t b = (uint64_t)__double_as_longlong(a) & 0x7fffffffffffffffULL;
    int be = (int)(b >> 52);
    if (be == 0) {
        double s = __longlong_as_double((long long)b) * 18014398509481984.0; /* 2^54 */
        be = (int)(((uint64_t)__double_as_longlong(s)) >> 52) - 54;
    }
    return be - 1022;
}

__device__ __forceinline__ double ldexp2(double x, int k)
{
    int k1 = k / 2;
    int k2 = k - k1;
    return (x * st_pow2i(k1)) * st_pow2i(k2);
}

/* Quantises one deposit component; returns 0 for zero, non-finite or out-of-range values
 * (the latter two are counted in `ovf`).  Updates the running max exponent. */
__device__ __forceinline__ long long quantize(double dv, int L, int cap, int& emax,
                                              unsigned& ovf)
{
    if (dv == 0.0) return 0;
    if (!isfinite(dv)) {
        ++ovf;
        return 0;
    }
    int e = exp_of(dv);
    emax = max(emax, e);
    if (e - L > cap) {
        ++ovf;
        return 0;
    }
    return __double2ll_rn(ldexp2(dv, -L));
}

template <int DEP>
__device__ __forceinline__ void deposit_direct(const double dep[3], int64_t cell0,
                                               unsigned long long* acc, double* src, int L,
                                               int cap, int& emax, unsigned& ovf)
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (DEP == DEP_ATOMIC) {
            if (dep[c] != 0.0) atomicAdd(src + 3 * cell0 + c, dep[c]);
        } else {
            long long q = quantize(dep[c], L, cap, emax, ovf);
            if (DEP == DEP_DET1) {
                if (q) atomicAdd(acc + 3 * cell0 + c, (unsigned long long)q);
            } else if (DEP == DEP_DET2) {
                if (q) {
                    atomicAdd(acc + 2 * (3 * cell0 + c), (unsigned long long)(q >> 32));
                    atomicAdd(acc + 2 * (3 * cell0 + c) + 1,
                              (unsigned long long)q & 0xffffffffULL);
                }
            }
        }
    }
}

/* Inclusive scan over the lane's run of equal keys (runs are contiguous lane ranges). */
template <class T>
__device__ __forceinline__ T seg_scan(T v, int lane, int segstart)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        T t = __shfl_up_sync(FULL_MASK, v, off);
        if (lane - off >= segstart) v += t;
    }
    return v;
}

/* ------------------------------------------------------------------------------------ */
/* the step kernel                                                                      */
/* ------------------------------------------------------------------------------------ */

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

template <class T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
template <class T>
__device__ __forceinline__ void st_stream(T* p, T v) { __stcs(p, v); }

template <class P, class V, int DEP>
__global__ void __launch_bounds__(256) k_step(const StepArgs<P, V> a)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const MeshK<P>& mesh = a.mesh;
    const PhysK<V>& ph = a.phys;
    const P dtP = a.dtP;
    const V dtV = a.dtV;
    const V fs = a.fscale;

    for (int64_t tile = warp0; tile < a.total_tiles; tile += nwarps) {
        const int c = (a.nclouds == 1) ? 0 : find_cloud(a, tile);
        const CloudK<P, V>* cl = a.clouds + c;
        const int64_t n = __ldg(&cl->n);
        const int64_t i = (tile - __ldg(&cl->tile0)) * 32 + lane;
        const bool active = i < n;
        CloudCtl* ctl = a.ctl + c;
        const int L = (DEP == DEP_DET1 || DEP == DEP_DET2) ? ctl->L : 0;
        const int cap = (DEP == DEP_DET1 || DEP == DEP_DET2) ? ctl->H + QUANT_GROWTH_BITS : 0;
        unsigned long long* acc = (DEP == DEP_DET1 || DEP == DEP_DET2) ? cl->acc : nullptr;
        double* src = (DEP == DEP_ATOMIC) ? cl->src : nullptr;

        int emax = EXP_NONE;
        unsigned ovf = 0;
        bool lost = false;
        int32_t key = -1;            /* 0-based cell of the final deposit */
        double dep[3] = {0.0, 0.0, 0.0};

        if (active) {
            P pos[3], posNew[3];
            V vel[3], velNew[3];
            P* xp = cl->x;
            P* yp = cl->y;
            P* zp = cl->z;
            V* up = cl->u;
            V* vp = cl->v;
            V* wp = cl->w;
            pos[0] = ld_stream(xp + i);
            pos[1] = ld_stream(yp + i);
            pos[2] = ld_stream(zp + i);
            vel[0] = ld_stream(up + i);
            vel[1] = ld_stream(vp + i);
            vel[2] = ld_stream(wp + i);
            const V d = ld_stream(cl->d + i) * ph.dscale;
            /* mᵈ/ρᶜ = ρᵈ/ρᶜ·π·⌀³/6 (A:1280) */
            const V mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;
            /* drag factor 18 μ Δt/(ρᵈ ⌀²) (A:1294), times the drag multiplier */
            const V f = ((((V)18 * ph.mu) * dtV) / (ph.rho_d * (d * d))) * ph.alpha;

            bool bad = false;
            LocK l0 = locate(mesh, pos[0], pos[1], pos[2], bad);         /* A:1286 */
            if (bad || l0.part != 1) {
                lost = true;
            } else {
                int32_t posI = l0.posI;
                const V* Uc = a.U + 3 * (int64_t)(posI - 1);             /* A:1288 */
                V uc[3] = {__ldg(Uc) * fs, __ldg(Uc + 1) * fs, __ldg(Uc + 2) * fs};
                V state0[3] = {vel[0], vel[1], vel[2]};                 /* A:1289 */
                for (int t = 1; t <= ph.nsub; ++t) {
                    if (ph.drag == 0) {
#pragma unroll
                        for (int k = 0; k < 3; ++k)                      /* A:1295 */
                            velNew[k] = (vel[k] + f * uc[k]) / ((V)1 + f);
                    } else {
                        V du[3];
#pragma unroll
                        for (int k = 0; k < 3; ++k) du[k] = uc[k] - vel[k];
                        V mag = st_sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2]);
                        V Re = (mag * d) / ph.nu;
                        V pw;
                        if (sizeof(V) == 4) pw = (V)st_pow0687f((float)Re);
                        else pw = (V)st_pow0687((double)Re);
                        V g = f * ((V)1 + (V)0.15 * pw);
#pragma unroll
                        for (int k = 0; k < 3; ++k) velNew[k] = vel[k] + g * du[k];
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) posNew[k] = pos[k] + (P)velNew[k] * dtP;  /* A:1296 */

                    LocK ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);      /* A:1303 */
                    if (bad) { lost = true; break; }
                    if (ln.posI != posI || ln.part != 1) {                               /* A:1306 */
                        const bool bx = (ln.I < 0) || (ln.I >= mesh.N[0]);
                        const bool by = (ln.J < 0) || (ln.J >= mesh.N[1]);
                        const bool bz = (ln.K < 0) || (ln.K >= mesh.N[2]);
                        /* hold position, mirror the old velocity, state0 -= 2 vel (A:1313-1329) */
                        if (bx) { posNew[0] = pos[0]; velNew[0] = -vel[0]; state0[0] -= (V)2 * vel[0]; }
                        if (by) { posNew[1] = pos[1]; velNew[1] = -vel[1]; state0[1] -= (V)2 * vel[1]; }
                        if (bz) { posNew[2] = pos[2]; velNew[2] = -vel[2]; state0[2] -= (V)2 * vel[2]; }
                        if (bx || by || bz) {                                            /* A:1333-1335 */
                            ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);
                            if (bad) { lost = true; break; }
                        }
                        if (t != ph.nsub && ln.posI != posI) {                           /* A:1342-1348 */
                            if (ln.part != 1 || ln.posI < 1 || ln.posI > mesh.nCells) {
                                lost = true;
                                break;
                            }
                            double di[3];
#pragma unroll
                            for (int k = 0; k < 3; ++k) di[k] = (double)(mB * (state0[k] - velNew[k]));
                            if (DEP == DEP_PROBE) {
#pragma unroll
                                for (int k = 0; k < 3; ++k)
                                    if (di[k] != 0.0 && isfinite(di[k])) emax = max(emax, exp_of(di[k]));
                            } else {
                                deposit_direct<DEP>(di, (int64_t)(posI - 1), acc, src, L, cap, emax, ovf);
                            }
#pragma unroll
                            for (int k = 0; k < 3; ++k) state0[k] = velNew[k];
                            const V* Un = a.U + 3 * (int64_t)(ln.posI - 1);
                            uc[0] = __ldg(Un) * fs;
                            uc[1] = __ldg(Un + 1) * fs;
                            uc[2] = __ldg(Un + 2) * fs;
                            posI = ln.posI;
                        }
                    }
#pragma unroll
                    for (int k = 0; k < 3; ++k) { vel[k] = velNew[k]; pos[k] = posNew[k]; }
                }
                if (!lost) {
                    if (DEP != DEP_PROBE) {                                             /* A:1355-1360 */
                        st_stream(xp + i, posNew[0]);
                        st_stream(yp + i, posNew[1]);
                        st_stream(zp + i, posNew[2]);
                        st_stream(up + i, velNew[0]);
                        st_stream(vp + i, velNew[1]);
                        st_stream(wp + i, velNew[2]);
                    }
                    key = posI - 1;                                                      /* A:1361 */
#pragma unroll
                    for (int k = 0; k < 3; ++k) dep[k] = (double)(mB * (state0[k] - velNew[k]));
                }
            }
        }

        /* ---- final deposit: one per parcel into posI ---- */
        if (DEP == DEP_PROBE) {
            if (key >= 0) {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (dep[k] != 0.0 && isfinite(dep[k])) emax = max(emax, exp_of(dep[k]));
            }
        } else if (DEP == DEP_ATOMIC) {
            if (key >= 0) deposit_direct<DEP_ATOMIC>(dep, key, acc, src, L, cap, emax, ovf);
        } else {
            long long q[3] = {0, 0, 0};
            if (key >= 0) {
#pragma unroll
                for (int k = 0; k < 3; ++k) q[k] = quantize(dep[k], L, cap, emax, ovf);
            }
            /* runs of equal cells among the 32 consecutive parcels of this tile */
            const int prev = __shfl_up_sync(FULL_MASK, key, 1);
            const bool head = (lane == 0) || (prev != key);
            const unsigned heads = __ballot_sync(FULL_MASK, head);
            const int segstart = 31 - __clz(heads & (FULL_MASK >> (31 - lane)));
            const bool tail = (lane == 31) || ((heads >> (lane + 1)) & 1u);
            if (DEP == DEP_DET1) {
#pragma unroll
                for (int k = 0; k < 3; ++k) q[k] = seg_scan(q[k], lane, segstart);
                if (tail && key >= 0) {
                    unsigned long long* p = acc + 3 * (int64_t)key;
#pragma unroll
                    for (int k = 0; k < 3; ++k)
                        if (q[k]) atomicAdd(p + k, (unsigned long long)q[k]);
                }
            } else {
                long long hi[3];
                unsigned long long lo[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    hi[k] = seg_scan(q[k] >> 32, lane, segstart);
                    lo[k] = seg_scan((unsigned long long)q[k] & 0xffffffffULL, lane, segstart);
                }
                if (tail && key >= 0) {
                    unsigned long long* p = acc + 6 * (int64_t)key;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        if (hi[k]) atomicAdd(p + 2 * k, (unsigned long long)hi[k]);
                        if (lo[k]) atomicAdd(p + 2 * k + 1, lo[k]);
                    }
                }
            }
        }

        /* ---- bookkeeping: scale tracker, lost parcels, range errors ---- */
        if (DEP != DEP_ATOMIC) {
            const int wmax = __reduce_max_sync(FULL_MASK, emax);
            if (lane == 0 && wmax != EXP_NONE) atomicMax(&ctl->emax, wmax);
        }
        const unsigned nlost = __popc(__ballot_sync(FULL_MASK, lost));
        const unsigned novf = __reduce_add_sync(FULL_MASK, ovf);
        if (lane == 0) {
            if (nlost) atomicAdd(&ctl->lost, (unsigned long long)nlost);
            if (novf && DEP != DEP_PROBE) atomicAdd(&ctl->overflow, (unsigned long long)novf);
        }
    }
}

template <class P, class V>
cudaError_t launch_step(const StepArgs<P, V>& a, int dep, int grid, int block, cudaStream_t s)
{
    switch (dep) {
    case DEP_DET1: k_step<P, V, DEP_DET1><<<grid, block, 0, s>>>(a); break;
    case DEP_DET2: k_step<P, V, DEP_DET2><<<grid, block, 0, s>>>(a); break;
    case DEP_ATOMIC: k_step<P, V, DEP_ATOMIC><<<grid, block, 0, s>>>(a); break;
    case DEP_PROBE: k_step<P, V, DEP_PROBE><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class P, class V>
int step_max_active_blocks(int dep, int block)
{
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (dep) {
    case DEP_DET1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_DET1>, block, 0); break;
    case DEP_DET2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_DET2>, block, 0); break;
    case DEP_ATOMIC: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_ATOMIC>, block, 0); break;
    case DEP_PROBE: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<P, V, DEP_PROBE>, block, 0); break;
    default: break;
    }
    return e == cudaSuccess ? nb : 0;
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
                                                  double* __restrict__ src, CloudCtl* ctl,
                                                  unsigned int* counter, int nclouds,
                                                  int64_t ncomp)
{
    const int c = blockIdx.y;
    const int L = ctl[c].L;
    unsigned long long* a = acc + (int64_t)c * ncomp * LIMBS;
    double* s = src + (int64_t)c * ncomp;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ncomp; j += stride) {
        double v;
        if (LIMBS == 1) {
            v = (double)(long long)a[j];
            a[j] = 0ULL;
        } else {
            long long hi = (long long)a[2 * j];
            unsigned long long lo = a[2 * j + 1];
            hi += (long long)(lo >> 32);
            lo &= 0xffffffffULL;
            v = (double)hi * 4294967296.0 + (double)lo;
            a[2 * j] = 0ULL;
            a[2 * j + 1] = 0ULL;
        }
        __stcs(s + j, ldexp2(v, L));
    }
    /* the last block to finish moves every cloud to the scale of its largest deposit */
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

cudaError_t launch_finalize(int limbs, unsigned long long* acc, double* src, CloudCtl* ctl,
                            unsigned int* counter, int nclouds, int64_t ncomp, int grid_x,
                            cudaStream_t s)
{
    dim3 grid(grid_x, nclouds);
    if (limbs == 1) k_finalize<1><<<grid, 256, 0, s>>>(acc, src, ctl, counter, nclouds, ncomp);
    else k_finalize<2><<<grid, 256, 0, s>>>(acc, src, ctl, counter, nclouds, ncomp);
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

cudaError_t launch_set_scale(CloudCtl* ctl, int nclouds, cudaStream_t s)
{
    k_set_scale<<<(nclouds + 127) / 128, 128, 0, s>>>(ctl, nclouds);
    return cudaGetLastError();
}

__global__ void k_zero_f64(double* p, int64_t n)
{
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x)
        p[j] = 0.0;
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
