/*
 * st_ring.cuh -- the shared-memory ring that streams a cloud's parcel state through the SMs
 * (used by the hex step kernel, st_ring.cu, and the tet step kernel, st_tet.cu).
 *
 * One block per SM.  The cloud's parcels are cut into block tiles of BT consecutive
 * parcels; tile t belongs to block t mod grid.  A producer warp streams each tile's state
 * arrays (x, y, z, u, v, w, d and, on tet meshes, the owning tet: 4-8 KB each) from HBM into
 * a stage of a RING_NS-deep ring in shared memory with 1-D bulk copies (cp.async.bulk, no
 * multicast: every source is this GPU's own memory) that complete on the stage's "full"
 * mbarrier.  The consumer warps step the tile out of shared memory, write the new state back
 * into the stage and arrive on its "empty" mbarrier; the producer then writes the stage back
 * to HBM with bulk stores and, once they have read it, refills the stage with a tile RING_NS
 * ahead.  The loads of up to RING_NS - 1 tiles are in flight while a tile is stepped,
 * independent of how many warps are resident, and the consumers spend no instructions on
 * global addressing.  The last block also steps the ragged end of the cloud (fewer than
 * BT parcels) with direct loads and stores.  The tile size and the number of consumer warps
 * are a RingShape per kernel.
 *
 * Every wait on an mbarrier gives up after about a second of clock cycles, sets the cloud's
 * fault word and lets the block drain (the producer waits, again bounded, for its own copies
 * in flight) so the host sees an error instead of a hung device.
 */
#ifndef ST_RING_CUH
#define ST_RING_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "st_device.cuh"

namespace st {

constexpr long long RING_WAIT_CYCLES = 2000000000LL;        /* about 1 s at 1.9 GHz        */
constexpr int RING_MAX_NS = 4;

/* The shape of a ring block: BT parcels per block tile, CONS consumer warps (one producer
 * warp more), SPW 32-parcel slices per consumer warp and tile.  BT * 4 bytes must be a
 * multiple of 16 (bulk copies start on 16-byte boundaries). */
template <int BT_, int CONS_>
struct RingShape {
    static constexpr int BT = BT_;
    static constexpr int CONS = CONS_;
    static constexpr int THREADS = 32 * (CONS_ + 1);
    static constexpr int SPW = BT_ / (32 * CONS_);
    static_assert(SPW * 32 * CONS_ == BT_, "tile split");
    static_assert((BT_ * 4) % 16 == 0, "16-byte tiles");
};

template <class S, class P, class V, bool CELL>
struct RingGeom {
    static constexpr uint32_t SP = S::BT * sizeof(P);       /* bytes of one position array */
    static constexpr uint32_t SV = S::BT * sizeof(V);       /* bytes of one velocity array */
    static constexpr uint32_t SC = CELL ? S::BT * 4 : 0;    /* the owning-tet array        */
    static constexpr uint32_t STAGE = 3 * SP + 4 * SV + SC;
    static constexpr int NS = (RING_MAX_NS * STAGE <= 200u * 1024u)
                                  ? RING_MAX_NS
                                  : (int)((200u * 1024u) / STAGE);
    static constexpr uint32_t SMEM = NS * STAGE;
    static_assert(NS >= 2, "at least two stages");
    static_assert(SMEM <= 227u * 1024u, "shared memory");
};

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

/* The pipeline-wait limit of a launch from its wait_cycles argument: |wait_cycles| when
 * non-zero, else RING_WAIT_CYCLES.  A negative value also asks for the failure-detection
 * test: the consumers first wait on a barrier that nothing completes. */
__device__ __forceinline__ long long ring_wait_limit(long long cycles)
{
    return cycles > 0 ? cycles : cycles < 0 ? -cycles : RING_WAIT_CYCLES;
}

/* Waits until the phase of parity `parity` of the barrier has completed; false when that
 * has not happened within ring_wait_limit(wait_cycles) SM clock cycles (the limit is worked
 * out only once the first try has failed). */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long wait_cycles = 0)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long limit = ring_wait_limit(wait_cycles);
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
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

/* The state arrays of a ring tile, in shared memory (a stage) or in global memory (the
 * ragged end); `cell` only on tet meshes. */
template <class P, class V>
struct RingArrays {
    P* x;
    P* y;
    P* z;
    V* u;
    V* v;
    V* w;
    const V* d;
    int32_t* cell;
};

template <class P, class V>
__device__ __forceinline__ RingArrays<P, V> ring_global(const CloudK<P, V>& c, int64_t off)
{
    return {c.x + off, c.y + off, c.z + off, c.u + off, c.v + off, c.w + off, c.d + off,
            c.cell ? c.cell + off : nullptr};
}

template <class S, class P, class V, bool CELL>
__device__ __forceinline__ RingArrays<P, V> ring_stage(unsigned char* stage)
{
    P* x = reinterpret_cast<P*>(stage);
    V* u = reinterpret_cast<V*>(x + 3 * S::BT);
    V* d = u + 3 * S::BT;
    return {x, x + S::BT, x + 2 * S::BT, u, u + S::BT, u + 2 * S::BT, d,
            CELL ? reinterpret_cast<int32_t*>(d + S::BT) : nullptr};
}

/* The producer (one thread): loads tiles into the ring, writes stepped tiles back. */
template <class S, class P, class V, bool CELL>
__device__ __forceinline__ void ring_producer(const CloudK<P, V>& cl, CloudCtl* ctl, int64_t cnt,
                                              int64_t blk, int64_t nblk, uint32_t sbase,
                                              uint32_t full0, uint32_t empty0,
                                              long long wait_cycles)
{
    using R = RingGeom<S, P, V, CELL>;
    const uint64_t pol = policy_evict_first();
    int64_t issued = 0;
    bool ok = true;
    for (int64_t k = 0; k < cnt + R::NS; ++k) {
        if (k >= R::NS) {
            /* tile j = k - NS has been stepped in stage j mod NS: write it back */
            const int64_t j = k - R::NS;
            const int s = (int)(j % R::NS);
            if (!mbar_wait(empty0 + 8 * s, (uint32_t)((j / R::NS) & 1), wait_cycles)) {
                ok = false;
                break;
            }
            const int64_t p0 = (blk + j * nblk) * S::BT;
            const uint32_t st = sbase + s * R::STAGE;
            bulk_store(cl.x + p0, st, R::SP, pol);
            bulk_store(cl.y + p0, st + R::SP, R::SP, pol);
            bulk_store(cl.z + p0, st + 2 * R::SP, R::SP, pol);
            bulk_store(cl.u + p0, st + 3 * R::SP, R::SV, pol);
            bulk_store(cl.v + p0, st + 3 * R::SP + R::SV, R::SV, pol);
            bulk_store(cl.w + p0, st + 3 * R::SP + 2 * R::SV, R::SV, pol);
            if (CELL) bulk_store(cl.cell + p0, st + 3 * R::SP + 4 * R::SV, R::SC, pol);
            bulk_commit();
        }
        if (k < cnt) {
            const int s = (int)(k % R::NS);
            /* the stage is free once the stores of its previous tile have read it */
            if (k >= R::NS) bulk_wait_read_all();
            const int64_t p0 = (blk + k * nblk) * S::BT;
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
            if (CELL) bulk_load(st + 3 * R::SP + 4 * R::SV, cl.cell + p0, R::SC, fb, pol);
            issued = k + 1;
        }
    }
    bulk_wait_all();
    if (!ok) {
        ring_fault(ctl, 1);
        /* the loads still in flight write into this block's shared memory: wait (bounded
         * by RING_WAIT_CYCLES, whatever the launch's limit) for the last one issued into
         * every stage before the block may exit */
        for (int s = 0; s < R::NS && s < issued; ++s) {
            const int64_t last = s + ((issued - 1 - s) / R::NS) * R::NS;
            mbar_wait(full0 + 8 * s, (uint32_t)((last / R::NS) & 1));
        }
    }
}

/* The block's part of the ring: barrier set-up, then the producer warp streams the block's
 * tiles and the consumer warps call step.run<false>(stage arrays, j0, S::BT) per tile and,
 * in the last block, step.run<true>(global arrays, j0, n mod S::BT) for the ragged end
 * (j0 = the lane's first parcel of the warp's slices).  Returns false in the producer warp,
 * which must then return without touching barrier 1 (the consumers' named barrier).
 * wait_cycles: the limit of the pipeline waits (ring_wait_limit). */
template <class S, class P, class V, bool CELL, class Step>
__device__ __forceinline__ bool ring_block(const CloudK<P, V>& cl, CloudCtl* ctl, Step& step,
                                           long long wait_cycles)
{
    using R = RingGeom<S, P, V, CELL>;
    extern __shared__ __align__(128) unsigned char ring_smem[];
    __shared__ __align__(8) unsigned long long ring_bars[2 * RING_MAX_NS + 1];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t n = cl.n;
    const int64_t nfull = n / S::BT;
    const int64_t nblk = gridDim.x;
    const int64_t blk = blockIdx.x;
    const int64_t cnt = blk < nfull ? (nfull - 1 - blk) / nblk + 1 : 0;
    const uint32_t sbase = smem_u32(ring_smem);
    const uint32_t full0 = smem_u32(ring_bars);
    const uint32_t empty0 = full0 + 8 * R::NS;
    const uint32_t never = full0 + 8 * (2 * RING_MAX_NS);   /* the test's barrier: no arrivals */
    if (threadIdx.x == 0) {
        for (int s = 0; s < R::NS; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, S::CONS);
        }
        mbar_init(never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == S::CONS) {
        if (lane == 0)
            ring_producer<S, P, V, CELL>(cl, ctl, cnt, blk, nblk, sbase, full0, empty0,
                                         wait_cycles);
        return false;
    }
    const int j0 = warp * (S::SPW * 32) + lane;
    bool ok = true;
    if (wait_cycles < 0) ok = __all_sync(FULL_MASK, mbar_wait(never, 0, wait_cycles));
    for (int64_t k = 0; ok && k < cnt; ++k) {
        const int s = (int)(k % R::NS);
        /* every lane waits; the warp goes on only if all of them saw the stage arrive */
        ok = __all_sync(FULL_MASK,
                        mbar_wait(full0 + 8 * s, (uint32_t)((k / R::NS) & 1), wait_cycles));
        if (!ok) break;
        step.template run<false>(ring_stage<S, P, V, CELL>(ring_smem + (size_t)s * R::STAGE), j0,
                                 (int64_t)S::BT);
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * s);
    }
    if (!ok) ring_fault(ctl, 2);
    /* the ragged end of the cloud: the last block, straight from global memory */
    if (ok && blk == nblk - 1 && n > nfull * S::BT)
        step.template run<true>(ring_global(cl, nfull * S::BT), j0, n - nfull * S::BT);
    return true;
}

/* The largest deposit exponent of a ring block (thread 0 clears it before ring_block
 * synchronises the block). */
__shared__ int s_ring_emax;

__device__ __forceinline__ void ring_emax_init()
{
    if (threadIdx.x == 0) s_ring_emax = EXP_NONE;
}

/* barrier among the consumer warps of a ring block (the producer warp has returned) */
template <class S>
__device__ __forceinline__ void ring_consumers_sync()
{
    asm volatile("bar.sync 1, %0;" ::"n"(S::CONS * 32) : "memory");
}

/* After flush_ctl has put every consumer warp's largest exponent into s_ring_emax: a
 * barrier among the consumer warps, then thread 0 adds the block's maximum to the cloud's
 * exponent word, one device-scope atomic per block instead of one per warp on that single
 * word (hex step kernel 0.1933 -> 0.1866 ms per launch on the 1e7-parcel step).  No memory
 * fence (__threadfence or __threadfence_block): one in these kernels, even a block-scope one
 * that ordered shared-memory counts in place of the barrier, made them about 45 % slower,
 * also where it never ran. */
template <class S>
__device__ __forceinline__ void ring_emax_flush(CloudCtl* ctl)
{
    ring_consumers_sync<S>();
    if (threadIdx.x == 0 && s_ring_emax != EXP_NONE) atomicMax(&ctl->emax, s_ring_emax);
}

}  // namespace st

#endif
