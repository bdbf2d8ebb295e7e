/*
 * st_ring.cu -- the parcel step of one cloud as a persistent shared-memory ring, for sm_100a.
 *
 * One block per SM.  The cloud's parcels are cut into block tiles of RING_BT consecutive
 * parcels; tile t belongs to block t mod grid.  A producer warp streams each tile's seven
 * state arrays (x, y, z, u, v, w, d: 4-8 KB each) from HBM into a stage of a RING_NS-deep
 * ring in shared memory with 1-D bulk copies (cp.async.bulk, no multicast: every source is
 * this GPU's own memory) that complete on the stage's "full" mbarrier.  Sixteen consumer
 * warps step the tile out of shared memory -- two 32-parcel slices per warp, their cell
 * velocity gathers issued together -- write the new positions and velocities back into the
 * stage and arrive on its "empty" mbarrier; the producer then writes the stage back to HBM
 * with bulk stores and, once they have read it, refills the stage with a tile RING_NS ahead.
 * The loads of up to RING_NS - 1 tiles are in flight while a tile is stepped, independent of
 * how many warps are resident, and the consumers spend no instructions on global addressing.
 * The last block also steps the ragged end of the cloud (fewer than RING_BT parcels) with
 * direct loads and stores.
 *
 * Arithmetic, deposit and bookkeeping are those of the warp-tile kernel (st_step.cuh,
 * st_device.cuh): positions, velocities, cells and the fixed-point source are bit-identical.
 * Every wait on an mbarrier gives up after about a second of clock cycles, sets the cloud's
 * fault word and lets the block drain (the producer waits, again bounded, for its own copies
 * in flight) so the host sees an error instead of a hung device.
 *
 * Reference: A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 *   evolve_on_device!  A:1258-1269     evolve_particle!  A:1271-1365
 */
#include <cstdint>
#include <atomic>
#include <cuda_runtime.h>

#include "st_step.cuh"

namespace st {

#ifndef ST_RING_BT
#define ST_RING_BT 1024
#endif
#ifndef ST_RING_CONSUMERS
#define ST_RING_CONSUMERS 16
#endif
#ifndef ST_RING_MAX_NS
#define ST_RING_MAX_NS 4
#endif
constexpr int RING_BT = ST_RING_BT;                         /* parcels per block tile      */
constexpr int RING_CONSUMERS = ST_RING_CONSUMERS;           /* consumer warps per block    */
constexpr int RING_THREADS = 32 * (RING_CONSUMERS + 1);     /* + one producer warp         */
constexpr int RING_SPW = RING_BT / (32 * RING_CONSUMERS);   /* slices per warp and tile    */
constexpr long long RING_WAIT_CYCLES = 2000000000LL;        /* about 1 s at 1.9 GHz        */
constexpr int RING_MAX_NS = ST_RING_MAX_NS;

template <class P, class V>
struct RingGeom {
    static constexpr uint32_t SP = RING_BT * sizeof(P);     /* bytes of one position array */
    static constexpr uint32_t SV = RING_BT * sizeof(V);     /* bytes of one velocity array */
    static constexpr uint32_t STAGE = 3 * SP + 4 * SV;
    static constexpr int NS = (RING_MAX_NS * STAGE <= 200u * 1024u)
                                  ? RING_MAX_NS
                                  : (int)((200u * 1024u) / STAGE);
    static constexpr uint32_t SMEM = NS * STAGE;
};
static_assert(RING_SPW * 32 * RING_CONSUMERS == RING_BT, "tile split");
static_assert(RingGeom<double, double>::SMEM <= 227u * 1024u, "shared memory");
static_assert(RingGeom<double, double>::NS >= 2, "at least two stages");

/* ------------------------------------------------------------------------------------ */
/* mbarrier and bulk-copy primitives (PTX)                                              */
/* ------------------------------------------------------------------------------------ */

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

/* Waits until the phase of parity `parity` of the barrier has completed; false when that
 * has not happened within RING_WAIT_CYCLES. */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > RING_WAIT_CYCLES) return false;
    return true;
}

__device__ __forceinline__ uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

/* global -> shared, completion counted in bytes on `bar` */
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar, uint64_t pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(pol)
        : "memory");
}

/* shared -> global, tracked by bulk groups of the issuing thread */
__device__ __forceinline__ void bulk_store(void* dst, uint32_t src, uint32_t bytes, uint64_t pol)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group.L2::cache_hint [%0], [%1], %2, %3;"
                 ::"l"(dst), "r"(src), "r"(bytes), "l"(pol)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all()
{
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

/* makes this thread's shared-memory writes visible to the bulk copies (async proxy) */
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void ring_fault(CloudCtl* ctl, int code)
{
    atomicOr(reinterpret_cast<unsigned int*>(&ctl->fault), (unsigned int)code);
}

/* ------------------------------------------------------------------------------------ */
/* consumer: RING_SPW slices of 32 parcels                                               */
/* ------------------------------------------------------------------------------------ */

template <bool GLOBAL, class T>
__device__ __forceinline__ T ring_ld(const T* p)
{
    if constexpr (GLOBAL) return ld_stream(p);
    else return *p;
}

template <bool GLOBAL, class T>
__device__ __forceinline__ void ring_st(T* p, T v)
{
    if constexpr (GLOBAL) st_stream(p, v);
    else *p = v;
}

/* Steps parcels j0, j0 + 32, ... (RING_SPW of them, those below nvalid) of the arrays: the
 * state of every slice is read and its cell velocity gathered first, then each slice is
 * stepped, written back and its deposits reduced (the warp-tile kernel's phases). */
template <class P, class V, int DEP, bool ONE, bool GLOBAL>
__device__ __forceinline__ void ring_slices(const StepArgs<P, V>& a, P* xs, P* ys, P* zs, V* us,
                                            V* vs, V* ws, const V* ds, int j0, int64_t nvalid,
                                            unsigned long long* acc, double* src,
                                            const Quant& qp, int lane, AmaxT<V>& amax,
                                            unsigned& ovf, unsigned& nlost)
{
    P X[RING_SPW], Y[RING_SPW], Z[RING_SPW];
    V Uv[RING_SPW], Vv[RING_SPW], Wv[RING_SPW], D[RING_SPW];
    int32_t pI[RING_SPW];
    V Ur[RING_SPW][3];
#pragma unroll
    for (int s = 0; s < RING_SPW; ++s) {
        const int j = j0 + 32 * s;
        pI[s] = 0;
        if (!GLOBAL || j < nvalid) {
            X[s] = ring_ld<GLOBAL>(xs + j);
            Y[s] = ring_ld<GLOBAL>(ys + j);
            Z[s] = ring_ld<GLOBAL>(zs + j);
            Uv[s] = ring_ld<GLOBAL>(us + j);
            Vv[s] = ring_ld<GLOBAL>(vs + j);
            Wv[s] = ring_ld<GLOBAL>(ws + j);
            D[s] = ring_ld<GLOBAL>(ds + j);
            bool bad = false;
            LocK l0 = locate(a.mesh, X[s], Y[s], Z[s], bad);                  /* A:1286 */
            if (!bad && l0.part == 1) {
                pI[s] = l0.posI;
                const V* Uc = a.U + 3 * (int64_t)(l0.posI - 1);                /* A:1288 */
                Ur[s][0] = __ldg(Uc);
                Ur[s][1] = __ldg(Uc + 1);
                Ur[s][2] = __ldg(Uc + 2);
            } else {
                ++nlost;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < RING_SPW; ++s) {
        const int j = j0 + 32 * s;
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
                evolve_parcel<P, V, DEP>(a, pos, vel, D[s] * a.phys.dscale, pI[s], Ur[s], acc,
                                         src, qp, amax, ovf, lost, key, dep);
            }
            if (lost) {
                ++nlost;
                key = -1;
            } else {                                                          /* A:1355-1360 */
                ring_st<GLOBAL>(xs + j, pos[0]);
                ring_st<GLOBAL>(ys + j, pos[1]);
                ring_st<GLOBAL>(zs + j, pos[2]);
                ring_st<GLOBAL>(us + j, vel[0]);
                ring_st<GLOBAL>(vs + j, vel[1]);
                ring_st<GLOBAL>(ws + j, vel[2]);
            }
        }
        deposit_warp<DEP, V>(key, dep, acc, src, qp, lane, amax, ovf);
    }
}

/* ------------------------------------------------------------------------------------ */
/* producer                                                                             */
/* ------------------------------------------------------------------------------------ */

template <class P, class V>
__device__ __forceinline__ void ring_producer(const StepArgs<P, V>& a, int64_t cnt, int64_t blk,
                                              int64_t nblk, uint32_t sbase, uint32_t full0,
                                              uint32_t empty0)
{
    using R = RingGeom<P, V>;
    const CloudK<P, V>& cl = a.one;
    const uint64_t pol = policy_evict_first();
    int64_t issued = 0;
    bool ok = true;
    for (int64_t k = 0; k < cnt + R::NS; ++k) {
        if (k >= R::NS) {
            /* tile j = k - NS has been stepped in stage j mod NS: write it back */
            const int64_t j = k - R::NS;
            if (j >= cnt) continue;
            const int s = (int)(j % R::NS);
            if (!mbar_wait(empty0 + 8 * s, (uint32_t)((j / R::NS) & 1))) {
                ok = false;
                break;
            }
            const int64_t p0 = (blk + j * nblk) * RING_BT;
            const uint32_t st = sbase + s * R::STAGE;
            bulk_store(cl.x + p0, st, R::SP, pol);
            bulk_store(cl.y + p0, st + R::SP, R::SP, pol);
            bulk_store(cl.z + p0, st + 2 * R::SP, R::SP, pol);
            bulk_store(cl.u + p0, st + 3 * R::SP, R::SV, pol);
            bulk_store(cl.v + p0, st + 3 * R::SP + R::SV, R::SV, pol);
            bulk_store(cl.w + p0, st + 3 * R::SP + 2 * R::SV, R::SV, pol);
            bulk_commit();
        }
        if (k < cnt) {
            const int s = (int)(k % R::NS);
            /* the stage is free once the stores of its previous tile have read it */
            if (k >= R::NS) bulk_wait_read_all();
            const int64_t p0 = (blk + k * nblk) * RING_BT;
            const uint32_t st = sbase + s * R::STAGE;
            const uint32_t fb = full0 + 8 * s;
            mbar_expect_tx(fb, R::STAGE);
            bulk_load(st, cl.x + p0, R::SP, fb, pol);
            bulk_load(st + R::SP, cl.y + p0, R::SP, fb, pol);
            bulk_load(st + 2 * R::SP, cl.z + p0, R::SP, fb, pol);
            bulk_load(st + 3 * R::SP, cl.u + p0, R::SV, fb, pol);
            bulk_load(st + 3 * R::SP + R::SV, cl.v + p0, R::SV, fb, pol);
            bulk_load(st + 3 * R::SP + 2 * R::SV, cl.w + p0, R::SV, fb, pol);
            bulk_load(st + 3 * R::SP + 3 * R::SV, cl.d + p0, R::SV, fb, pol);
            issued = k + 1;
        }
    }
    bulk_wait_all();
    if (!ok) {
        ring_fault(a.ctl, 1);
        /* the loads still in flight write into this block's shared memory: wait (bounded)
         * for the last one issued into every stage before the block may exit */
        for (int s = 0; s < R::NS && s < issued; ++s) {
            const int64_t last = s + ((issued - 1 - s) / R::NS) * R::NS;
            mbar_wait(full0 + 8 * s, (uint32_t)((last / R::NS) & 1));
        }
    }
}

/* ------------------------------------------------------------------------------------ */
/* the kernel                                                                           */
/* ------------------------------------------------------------------------------------ */

template <class P, class V, int DEP, bool ONE>
__global__ void __launch_bounds__(RING_THREADS, 1) k_step_ring(const StepArgs<P, V> a)
{
    using R = RingGeom<P, V>;
    extern __shared__ __align__(128) unsigned char ring_smem[];
    __shared__ __align__(8) unsigned long long bars[2 * RING_MAX_NS];
    constexpr bool DET = (DEP == DEP_DET1 || DEP == DEP_DET2);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const CloudK<P, V>& cl = a.one;
    const int64_t n = cl.n;
    const int64_t nfull = n / RING_BT;
    const int64_t nblk = gridDim.x;
    const int64_t blk = blockIdx.x;
    const int64_t cnt = blk < nfull ? (nfull - 1 - blk) / nblk + 1 : 0;
    const uint32_t sbase = smem_u32(ring_smem);
    const uint32_t full0 = smem_u32(bars);
    const uint32_t empty0 = full0 + 8 * R::NS;
    if (threadIdx.x == 0) {
        for (int s = 0; s < R::NS; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, RING_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == RING_CONSUMERS) {
        if (lane == 0) ring_producer<P, V>(a, cnt, blk, nblk, sbase, full0, empty0);
        return;
    }

    Quant qp = {0.0, 0.0, 0.0f, 0.0f, 0, false};
    if (DET) qp = make_quant(a.ctl[0].L, a.ctl[0].H + QUANT_GROWTH_BITS);
    unsigned long long* const acc = DET ? cl.acc : nullptr;
    double* const src = (DEP == DEP_ATOMIC) ? cl.src : nullptr;
    AmaxT<V> amax = (V)0;
    unsigned ovf = 0, nlost = 0;
    const int j0 = warp * (RING_SPW * 32) + lane;
    bool ok = true;
    for (int64_t k = 0; k < cnt; ++k) {
        const int s = (int)(k % R::NS);
        /* every lane waits; the warp goes on only if all of them saw the stage arrive */
        ok = __all_sync(FULL_MASK, mbar_wait(full0 + 8 * s, (uint32_t)((k / R::NS) & 1)));
        if (!ok) break;
        unsigned char* stage = ring_smem + (size_t)s * R::STAGE;
        P* sx = reinterpret_cast<P*>(stage);
        P* sy = sx + RING_BT;
        P* sz = sy + RING_BT;
        V* su = reinterpret_cast<V*>(sz + RING_BT);
        V* sv = su + RING_BT;
        V* sw = sv + RING_BT;
        const V* sd = sw + RING_BT;
        ring_slices<P, V, DEP, ONE, false>(a, sx, sy, sz, su, sv, sw, sd, j0, RING_BT, acc, src,
                                           qp, lane, amax, ovf, nlost);
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * s);
    }
    if (!ok) ring_fault(a.ctl, 2);
    /* the ragged end of the cloud: the last block, straight from global memory */
    if (ok && blk == nblk - 1) {
        const int64_t p0 = nfull * RING_BT;
        if (n > p0)
            ring_slices<P, V, DEP, ONE, true>(a, cl.x + p0, cl.y + p0, cl.z + p0, cl.u + p0,
                                              cl.v + p0, cl.w + p0, cl.d + p0, j0, n - p0, acc,
                                              src, qp, lane, amax, ovf, nlost);
    }
    flush_ctl<DEP>(a.ctl, lane, amax, ovf, nlost);
}

/* ------------------------------------------------------------------------------------ */
/* host side                                                                            */
/* ------------------------------------------------------------------------------------ */

/* The shared-memory opt-in of one kernel instance on the current device, made once per
 * device (remembered in a bit mask per instance). */
template <class P, class V, int DEP, bool ONE>
static cudaError_t ring_attr()
{
    static std::atomic<unsigned long long> ready{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ULL << (dev & 63);
    if (ready.load() & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(k_step_ring<P, V, DEP, ONE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)RingGeom<P, V>::SMEM);
    if (e == cudaSuccess) ready.fetch_or(bit);
    return e;
}

template <class P, class V, int DEP, bool ONE>
static cudaError_t launch_ring_t(const StepArgs<P, V>& a, int nsm, cudaStream_t s)
{
    cudaError_t e = ring_attr<P, V, DEP, ONE>();
    if (e != cudaSuccess) return e;
    const int64_t nfull = a.one.n / RING_BT;
    int64_t grid = nfull < nsm ? nfull : nsm;
    if (grid < 1) grid = 1;
    k_step_ring<P, V, DEP, ONE><<<(int)grid, RING_THREADS, RingGeom<P, V>::SMEM, s>>>(a);
    return cudaGetLastError();
}

/* Makes every ring kernel instance of a precision launchable on the current device (called
 * when a handle is created, outside any stream capture). */
template <class P, class V>
cudaError_t ring_prepare()
{
    const cudaError_t r[6] = {ring_attr<P, V, DEP_DET1, true>(), ring_attr<P, V, DEP_DET1, false>(),
                              ring_attr<P, V, DEP_DET2, true>(), ring_attr<P, V, DEP_DET2, false>(),
                              ring_attr<P, V, DEP_ATOMIC, true>(),
                              ring_attr<P, V, DEP_ATOMIC, false>()};
    for (cudaError_t e : r)
        if (e != cudaSuccess) return e;
    return cudaSuccess;
}

template <class P, class V>
bool ring_eligible(const StepArgs<P, V>& a, int dep)
{
    if (a.nclouds != 1 || a.one.n <= 0) return false;
    if (dep != DEP_DET1 && dep != DEP_DET2 && dep != DEP_ATOMIC) return false;
    const void* p[7] = {a.one.x, a.one.y, a.one.z, a.one.u, a.one.v, a.one.w, a.one.d};
    for (const void* q : p)
        if (reinterpret_cast<uintptr_t>(q) % 16) return false;
    return true;
}

template <class P, class V>
cudaError_t launch_step_ring(const StepArgs<P, V>& a, int dep, int nsm, cudaStream_t s)
{
    if (a.nclouds != 1) return cudaErrorInvalidValue;
    const bool one = a.phys.nsub == 1;
    switch (dep) {
    case DEP_DET1: return one ? launch_ring_t<P, V, DEP_DET1, true>(a, nsm, s)
                              : launch_ring_t<P, V, DEP_DET1, false>(a, nsm, s);
    case DEP_DET2: return one ? launch_ring_t<P, V, DEP_DET2, true>(a, nsm, s)
                              : launch_ring_t<P, V, DEP_DET2, false>(a, nsm, s);
    case DEP_ATOMIC: return one ? launch_ring_t<P, V, DEP_ATOMIC, true>(a, nsm, s)
                                : launch_ring_t<P, V, DEP_ATOMIC, false>(a, nsm, s);
    default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_step_ring<float, float>(const StepArgs<float, float>&, int, int, cudaStream_t);
template cudaError_t launch_step_ring<double, float>(const StepArgs<double, float>&, int, int, cudaStream_t);
template cudaError_t launch_step_ring<double, double>(const StepArgs<double, double>&, int, int, cudaStream_t);
template cudaError_t ring_prepare<float, float>();
template cudaError_t ring_prepare<double, float>();
template cudaError_t ring_prepare<double, double>();
template bool ring_eligible<float, float>(const StepArgs<float, float>&, int);
template bool ring_eligible<double, float>(const StepArgs<double, float>&, int);
template bool ring_eligible<double, double>(const StepArgs<double, double>&, int);

}  // namespace st
