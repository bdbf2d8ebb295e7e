/*
 * st_ring.cu -- the parcel step of one cloud on the uniform hex mesh as a persistent
 * shared-memory ring (st_ring.cuh), for sm_100a.
 *
 * Twenty consumer warps step each 1280-parcel tile out of shared memory (FP64 velocities:
 * sixteen, 1024) -- two 32-parcel slices per warp, their cell velocity gathers issued
 * together -- and write the new positions and velocities back into the stage, which the
 * producer warp writes back to HBM with bulk stores.  Arithmetic, deposit and bookkeeping are those of the per-warp kernel (st_step.cuh,
 * st_device.cuh): positions, velocities, cells and the fixed-point source are bit-identical.
 *
 * Reference: A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 *   evolve_on_device!  A:1258-1269     evolve_particle!  A:1271-1365
 */
#include <cstdint>
#include <atomic>
#include <cuda_runtime.h>

#include "st_step.cuh"
#include "st_ring.cuh"


namespace st {

/* Ring shapes, two 32-parcel slices per consumer warp.  FP32 velocities (FP32 and mixed
 * precision, 40-byte parcels): 1280-parcel tiles and 20 consumer warps (21 warps: 96
 * registers, four 50 KB stages); measured on the 1e7-parcel step, 1024 x 16, 1152 x 18,
 * 1216 x 19 and 1280 x 20 took 0.1985, 0.1958, 0.1949 and 0.1943 ms.  FP64 velocities
 * (56-byte parcels): 1024-parcel tiles and 16 consumer warps, which keep three stages. */
#ifndef ST_RING_BT
#define ST_RING_BT 1280
#endif
#ifndef ST_RING_CONSUMERS
#define ST_RING_CONSUMERS 20
#endif
template <class V>
struct HexShapeOf {
    using type = RingShape<ST_RING_BT, ST_RING_CONSUMERS>;
};
template <>
struct HexShapeOf<double> {
    using type = RingShape<1024, 16>;
};
constexpr int RING_SPW = 2;
static_assert(HexShapeOf<float>::type::SPW == RING_SPW && HexShapeOf<double>::type::SPW == RING_SPW,
              "two slices per consumer warp");

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

/* The consumer work of the hex ring: ring_slices on the tile's arrays. */
template <class P, class V, int DEP, bool ONE>
struct HexRing {
    const StepArgs<P, V>& a;
    unsigned long long* acc;
    double* src;
    const Quant& qp;
    int lane;
    AmaxT<V>& amax;
    unsigned& ovf;
    unsigned& nlost;
    template <bool GLOBAL>
    __device__ __forceinline__ void run(const RingArrays<P, V>& r, int j0, int64_t nvalid)
    {
        ring_slices<P, V, DEP, ONE, GLOBAL>(a, r.x, r.y, r.z, r.u, r.v, r.w, r.d, j0, nvalid, acc,
                                            src, qp, lane, amax, ovf, nlost);
    }
};

template <class P, class V, int DEP, bool ONE>
__global__ void __launch_bounds__(HexShapeOf<V>::type::THREADS, 1)
    k_step_ring(const StepArgs<P, V> a)
{
    using HexShape = typename HexShapeOf<V>::type;
    constexpr bool DET = (DEP == DEP_DET1 || DEP == DEP_DET2);
    Quant qp = {0.0, 0.0, 0.0f, 0.0f, 0, false};
    if (DET) qp = make_quant(a.ctl[0].L, a.ctl[0].H + QUANT_GROWTH_BITS);
    AmaxT<V> amax = (V)0;
    unsigned ovf = 0, nlost = 0;
    const int lane = threadIdx.x & 31;
    HexRing<P, V, DEP, ONE> step{a, DET ? a.one.acc : nullptr,
                                 DEP == DEP_ATOMIC ? a.one.src : nullptr, qp, lane, amax, ovf,
                                 nlost};
    if (!ONE) pow_tab_fill();   /* ring_block synchronises the block before any step */
    ring_emax_init();
    if (!ring_block<HexShape, P, V, false>(a.one, a.ctl, step, a.wait_cycles)) return;
    flush_ctl<DEP>(a.ctl, lane, amax, ovf, nlost, DEP != DEP_ATOMIC ? &s_ring_emax : nullptr);
    if (DEP != DEP_ATOMIC) ring_emax_flush<HexShape>(a.ctl);
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
                             (int)RingGeom<typename HexShapeOf<V>::type, P, V, false>::SMEM);
    if (e == cudaSuccess) ready.fetch_or(bit);
    return e;
}

template <class P, class V, int DEP, bool ONE>
static cudaError_t launch_ring_t(const StepArgs<P, V>& a, int nsm, cudaStream_t s)
{
    using HexShape = typename HexShapeOf<V>::type;
    cudaError_t e = ring_attr<P, V, DEP, ONE>();
    if (e != cudaSuccess) return e;
    const int64_t nfull = a.one.n / HexShape::BT;
    int64_t grid = nfull < nsm ? nfull : nsm;
    if (grid < 1) grid = 1;
    k_step_ring<P, V, DEP, ONE>
        <<<(int)grid, HexShape::THREADS, RingGeom<HexShape, P, V, false>::SMEM, s>>>(a);
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
