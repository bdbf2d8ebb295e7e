/*
 * st_device.cuh -- device helpers shared by the step kernels of hex (st_kernels.cu) and
 * tetrahedral (st_tet.cu) meshes: IEEE helpers, the fixed-point deterministic deposit with
 * its warp-level run reduction, and the per-warp bookkeeping of the scale tracker.
 */
#ifndef ST_DEVICE_CUH
#define ST_DEVICE_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "st_internal.h"
#include "st_pow.h"

namespace st {

#ifndef FULL_MASK
#define FULL_MASK 0xffffffffu
#endif

__device__ __forceinline__ float st_sqrt(float v) { return __fsqrt_rn(v); }
__device__ __forceinline__ double st_sqrt(double v) { return __dsqrt_rn(v); }

__device__ __forceinline__ int32_t st_floor_int(float v) { return __float2int_rd(v); }
__device__ __forceinline__ int32_t st_floor_int(double v) { return __double2int_rd(v); }

/* Slip velocity u_c - v of one component, from the raw cell value Ur and the fluid factor
 * fs = fs_hi + fs_lo.  In mixed precision the product Ur*fs_hi stays exact inside one fma and
 * the low part of the FP64 factor is added, so the slip carries about one rounding of its
 * own size, also when the parcel has nearly relaxed to the carrier (|u - v| << |u|); the
 * FP32 and FP64 modes round u_c = U*fs to the velocity type first, as the reference does
 * (A:1288, A:1295). */
template <bool MIX, class V>
__device__ __forceinline__ V slip(V Ur, V fs_hi, V fs_lo, V vel)
{
    if constexpr (MIX) return __fmaf_rn(Ur, fs_hi, -vel) + Ur * fs_lo;
    else return Ur * fs_hi - vel;
}

/* x^0.687 in single precision (st_pow0687f) with its exponent factor, which depends only on
 * the binary exponent e of x, read from a table in shared memory.  The table is filled on
 * the device by st_pow0687f_efac itself, so the result is st_pow0687f's bit for bit.  A
 * kernel that calls pow0687f_tab fills the table (pow_tab_fill) and synchronises its block
 * first. */
constexpr int POW_TAB_EMIN = -150;   /* st_pow0687f_mant gives -149 <= e <= 128 */
constexpr int POW_TAB_N = 280;
__shared__ float2 s_pow_tab[POW_TAB_N];

__device__ __forceinline__ void pow_tab_fill()
{
    for (int i = threadIdx.x; i < POW_TAB_N; i += blockDim.x) {
        float q, s2k;
        st_pow0687f_efac(i + POW_TAB_EMIN, &q, &s2k);
        s_pow_tab[i] = make_float2(q, s2k);
    }
}

__device__ __forceinline__ float pow0687f_tab(float x)
{
    if (!(x > 0.0f)) return x != x ? x : 0.0f;
    if ((__float_as_uint(x) >> 23) == 0xffu) return x;   /* +inf */
    int e;
    const float p = st_pow0687f_mant(x, &e);
    const float2 qs = s_pow_tab[e - POW_TAB_EMIN];
    return (p * qs.x) * qs.y;
}

/* slip with the product of the raw cell value and the low part of the fluid factor given
 * (Ulo = Ur * fs_lo, formed once per cell by a multi-substep loop): the same value as slip */
template <bool MIX, class V>
__device__ __forceinline__ V slip_lo(V Ur, V fs_hi, V Ulo, V vel)
{
    if constexpr (MIX) return __fmaf_rn(Ur, fs_hi, -vel) + Ulo;
    else return Ur * fs_hi - vel;
}

/* floor(label, v) (A:668-670); values outside int32 mark the parcel as lost.  floor(v) lies
 * in [-2^31, 2^31) exactly when v does (both bounds are integers), so the range test is made
 * on v and one round-down conversion gives the label. */
template <class P>
__device__ __forceinline__ int32_t floor_label(P v, bool& bad)
{
    if (!(v >= (P)-2147483648.0 && v < (P)2147483648.0)) {
        bad = true;
        return 0;
    }
    return st_floor_int(v);
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

/* The running maximum of |deposit| is kept in the velocity precision (AmaxT<V>): every
 * deposit is a V value, so the maximum is exact in V and needs no conversion per deposit. */
template <class V>
using AmaxT = V;

/* largest finite |v| seen (probe pass) */
__device__ __forceinline__ void track_max(float v, float& amax)
{
    const float a = fabsf(v);
    if (a < __int_as_float(0x7f800000)) amax = fmaxf(amax, a);
}
__device__ __forceinline__ void track_max(double v, double& amax)
{
    const double a = fabs(v);
    if (a < __longlong_as_double(0x7ff0000000000000LL)) amax = fmax(amax, a);
}

/* Fixed-point parameters of one cloud for the current step: q = rint(dep * 2^-L), and a
 * deposit with |dep| >= 2^(cap+L) (i.e. frexp exponent - L > cap) does not fit.  Single
 * precision deposits are scaled in single precision when 2^-L and 2^(cap+L) are normal
 * floats: scaling by a power of two is exact, so the integer is the same as through FP64. */
struct Quant {
    double scale;   /* 2^-L, or 0 when 2^-L is not a normal double (then ldexp2 is used) */
    double thr;     /* 2^(cap+L) */
    float scale_f;  /* 2^-L as float, when `fast` */
    float thr_f;    /* 2^(cap+L) as float, when `fast` */
    int L;
    bool fast;
    float thr_small; /* 2^(SMALL_Q_BITS+L) as float when that is a normal float, else 0 */
};

/* Quantised deposits below 2^SMALL_Q_BITS in magnitude: a sum of up to four of them fits in
 * a 32-bit integer (the warp run reduction's 32-bit path). */
constexpr int SMALL_Q_BITS = 29;

__device__ __forceinline__ Quant make_quant(int L, int cap)
{
    Quant q;
    q.L = L;
    q.scale = (-L >= -1022 && -L <= 1023) ? st_pow2i(-L) : 0.0;
    q.thr = ldexp2(1.0, cap + L);
    q.fast = (-L >= -126 && -L <= 127) && (cap + L >= -126 && cap + L <= 127);
    q.scale_f = q.fast ? st_pow2if(-L) : 0.0f;
    q.thr_f = q.fast ? st_pow2if(cap + L) : 0.0f;
    q.thr_small = (q.fast && SMALL_Q_BITS + L >= -126 && SMALL_Q_BITS + L <= 127)
                      ? st_pow2if(SMALL_Q_BITS + L)
                      : 0.0f;
    return q;
}

/* Quantises one deposit component: 0 for zero, non-finite or out-of-range values (the
 * latter two are counted in `ovf`).  `amax` tracks the largest finite |dep| for the next
 * step's scale (max is order-independent, so the scale is reproducible). */
template <class A>
__device__ __forceinline__ long long quantize(double dv, const Quant& qp, A& amax,
                                              unsigned& ovf)
{
    const double a = fabs(dv);
    if (a == 0.0) return 0;
    /* exact for A = float: dv is then a float value */
    if (a < __longlong_as_double(0x7ff0000000000000LL)) amax = (A)fmax((double)amax, a);
    if (!(a < qp.thr)) {
        ++ovf;
        return 0;
    }
    const double x = qp.scale != 0.0 ? dv * qp.scale : ldexp2(dv, -qp.L);
    return __double2ll_rn(x);
}

__device__ __forceinline__ long long quantize(float dv, const Quant& qp, float& amax,
                                              unsigned& ovf)
{
    if (!qp.fast) return quantize((double)dv, qp, amax, ovf);
    const float a = fabsf(dv);
    if (a == 0.0f) return 0;
    if (a < __int_as_float(0x7f800000)) amax = fmaxf(amax, a);
    if (!(a < qp.thr_f)) {
        ++ovf;
        return 0;
    }
    return __float2ll_rn(dv * qp.scale_f);
}

/* The three components of one deposit.  In single precision with the fast scale: when
 * |d0| + |d1| + |d2| (rounded, which cannot fall below a power-of-two bound any single term
 * reaches) is below the range bound, every component is finite and in range, and each is
 * scaled and rounded directly, with the same integers and the same maximum as the
 * per-component path; otherwise (and in double precision) each component goes through
 * quantize, which counts what does not fit. */
__device__ __forceinline__ void quantize3(const float d[3], const Quant& qp, float& amax,
                                          unsigned& ovf, long long q[3])
{
    if (qp.fast) {
        const float a0 = fabsf(d[0]), a1 = fabsf(d[1]), a2 = fabsf(d[2]);
        if ((a0 + a1) + a2 < qp.thr_f) {
            amax = fmaxf(amax, fmaxf(fmaxf(a0, a1), a2));
#pragma unroll
            for (int k = 0; k < 3; ++k) q[k] = __float2ll_rn(d[k] * qp.scale_f);
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = quantize(d[k], qp, amax, ovf);
}

__device__ __forceinline__ void quantize3(const double d[3], const Quant& qp, double& amax,
                                          unsigned& ovf, long long q[3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = quantize(d[k], qp, amax, ovf);
}

template <int DEP, class V>
__device__ __forceinline__ void deposit_direct(const V dep[3], int64_t cell0,
                                               unsigned long long* acc, double* src,
                                               const Quant& qp, AmaxT<V>& amax, unsigned& ovf)
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (DEP == DEP_ATOMIC) {
            if (dep[c] != (V)0) atomicAdd(src + 3 * cell0 + c, (double)dep[c]);
        } else {
            long long q = quantize(dep[c], qp, amax, ovf);
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

#ifndef ST_SCAN_STEPS
#define ST_SCAN_STEPS 2
#endif
constexpr int SCAN_STEPS = ST_SCAN_STEPS;   /* 0..5 */
constexpr int SPAN = 1 << SCAN_STEPS;        /* lanes summed per emitted chunk */

/* Inclusive scan over the lane's run of equal keys, limited to SPAN lanes (runs are
 * contiguous lane ranges). */
template <class T>
__device__ __forceinline__ T seg_scan(T v, int lane, int segstart)
{
#pragma unroll
    for (int off = 1; off < SPAN; off <<= 1) {
        T t = __shfl_up_sync(FULL_MASK, v, off);
        if (lane - off >= segstart) v += t;
    }
    return v;
}

/* Streaming loads of the parcel arrays: evict-first (ld.global.cs) so that the cell arrays
 * keep L2, with a 256-byte L2 prefetch hint (each warp reads 128-256 contiguous bytes of an
 * array per tile; measured 0.5 % faster on the 1e7-parcel step than without the hint). */
__device__ __forceinline__ float ld_stream_(const float* p)
{
    float v;
    asm volatile("ld.global.cs.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_stream_(const double* p)
{
    double v;
    asm volatile("ld.global.cs.L2::256B.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ int32_t ld_stream_(const int32_t* p)
{
    int32_t v;
    asm volatile("ld.global.cs.L2::256B.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
template <class T>
__device__ __forceinline__ T ld_stream(const T* p) { return ld_stream_(p); }
template <class T>
__device__ __forceinline__ void st_stream(T* p, T v) { __stcs(p, v); }

/* Final deposits of 32 consecutive parcels (one per lane, key < 0 = none): runs of equal
 * cells are summed with a segmented warp scan and the last lane of each run adds the sum. */
template <int DEP, class V>
__device__ __forceinline__ void deposit_warp(int32_t key, const V dep[3],
                                             unsigned long long* acc, double* src,
                                             const Quant& qp, int lane, AmaxT<V>& amax,
                                             unsigned& ovf)
{
    if (DEP == DEP_PROBE) {
        if (key >= 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) track_max(dep[k], amax);
        }
        return;
    }
    if (DEP == DEP_ATOMIC) {
        if (key >= 0) deposit_direct<DEP_ATOMIC, V>(dep, key, acc, src, qp, amax, ovf);
        return;
    }
    const int prev = __shfl_up_sync(FULL_MASK, key, 1);
    const bool head = (lane == 0) || (prev != key);
    const unsigned heads = __ballot_sync(FULL_MASK, head);
    if constexpr (DEP == DEP_DET1 && sizeof(V) == 4) {
        /* 32-bit path: when every lane's deposit components quantise below 2^SMALL_Q_BITS
         * (|d0| + |d1| + |d2| below 2^(SMALL_Q_BITS+L), the bound argument of quantize3), the
         * integers are those of quantize3, a chunk of SPAN <= 4 lanes sums below 2^31, and the
         * run sums are formed in 32-bit registers: the same integers reach the accumulators. */
        int q32[3] = {0, 0, 0};
        bool small = key < 0;
        if (key >= 0) {
            const float a0 = fabsf((float)dep[0]), a1 = fabsf((float)dep[1]),
                        a2 = fabsf((float)dep[2]);
            if ((a0 + a1) + a2 < qp.thr_small) {
                amax = fmaxf(amax, fmaxf(fmaxf(a0, a1), a2));
#pragma unroll
                for (int k = 0; k < 3; ++k) q32[k] = __float2int_rn((float)dep[k] * qp.scale_f);
                small = true;
            }
        }
        static_assert(SPAN <= 4, "32-bit chunk sums");
        if (__all_sync(FULL_MASK, small)) {
            if (heads == 1u) {
                /* one cell for the whole warp: 16-bit halves, each sum exact in 32 bits */
                if (key >= 0) {
                    long long t[3];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const int shi = __reduce_add_sync(FULL_MASK, q32[k] >> 16);
                        const unsigned slo = __reduce_add_sync(FULL_MASK, (unsigned)q32[k] & 0xffffu);
                        t[k] = (long long)shi * 65536LL + (long long)slo;
                    }
                    if (lane == 0) {
                        unsigned long long* p = acc + 3 * (int64_t)key;
#pragma unroll
                        for (int k = 0; k < 3; ++k)
                            if (t[k]) atomicAdd(p + k, (unsigned long long)t[k]);
                    }
                }
                return;
            }
            const int segstart = 31 - __clz(heads & (FULL_MASK >> (31 - lane)));
            const bool tail = (lane == 31) || ((heads >> (lane + 1)) & 1u);
            const unsigned tails = __ballot_sync(FULL_MASK, tail);
            const int tailpos = lane + __ffs(tails >> lane) - 1;
            const bool emit = ((tailpos - lane) & (SPAN - 1)) == 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) q32[k] = seg_scan(q32[k], lane, segstart);
            if (emit && key >= 0) {
                unsigned long long* p = acc + 3 * (int64_t)key;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (q32[k]) atomicAdd(p + k, (unsigned long long)(long long)q32[k]);
            }
            return;
        }
    }
    long long q[3] = {0, 0, 0};
    if (key >= 0) quantize3(dep, qp, amax, ovf, q);
    if (DEP == DEP_DET1 && heads == 1u) {
        /* One cell for the whole warp (dense cells after a re-sort): exact full-warp
         * reductions replace the scan and lane 0 adds the sum.  With q = hi*2^32 + lo, the
         * sums of lo's two 16-bit halves stay below 2^21, and |sum of hi| <= 2^30 + 32 because
         * the headroom bounds the magnitudes of all of a step's deposits together by 2^62. */
        if (key >= 0) {
            long long t[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const unsigned lo = (unsigned)(unsigned long long)q[k];
                const long long shi = __reduce_add_sync(FULL_MASK, (int)(q[k] >> 32));
                const unsigned s0 = __reduce_add_sync(FULL_MASK, lo & 0xffffu);
                const unsigned s1 = __reduce_add_sync(FULL_MASK, lo >> 16);
                t[k] = shi * 4294967296LL + (long long)s0 + (long long)s1 * 65536LL;
            }
            if (lane == 0) {
                unsigned long long* p = acc + 3 * (int64_t)key;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (t[k]) atomicAdd(p + k, (unsigned long long)t[k]);
            }
        }
        return;
    }
    const int segstart = 31 - __clz(heads & (FULL_MASK >> (31 - lane)));
    const bool tail = (lane == 31) || ((heads >> (lane + 1)) & 1u);
    /* A scan of SCAN_STEPS steps sums runs in chunks of SPAN lanes: lane j holds the sum of
     * [max(run start, j - SPAN + 1), j]; the run's last lane and every SPAN-th lane before it
     * add their chunk, which covers the run exactly once. */
    const unsigned tails = __ballot_sync(FULL_MASK, tail);
    const int tailpos = lane + __ffs(tails >> lane) - 1;
    const bool emit = ((tailpos - lane) & (SPAN - 1)) == 0;
    if (DEP == DEP_DET1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) q[k] = seg_scan(q[k], lane, segstart);
        if (emit && key >= 0) {
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
        if (emit && key >= 0) {
            unsigned long long* p = acc + 6 * (int64_t)key;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (hi[k]) atomicAdd(p + 2 * k, (unsigned long long)hi[k]);
                if (lo[k]) atomicAdd(p + 2 * k + 1, lo[k]);
            }
        }
    }
}

/* Warp-aggregated bookkeeping for one cloud: largest deposit exponent, lost parcels and
 * range errors.  Called when a warp moves on to another cloud and at the end. */
template <int DEP, class A>
__device__ __forceinline__ void flush_ctl(CloudCtl* ctl, int lane, A& amax, unsigned& ovf,
                                          unsigned& lost, int* block_emax = nullptr)
{
    /* block_emax (shared memory): the warp's largest exponent goes there, and the kernel adds
     * the block's maximum to the control block once */
    if (DEP != DEP_ATOMIC) {
        const int e = amax > (A)0 ? exp_of((double)amax) : EXP_NONE;
        const int wmax = __reduce_max_sync(FULL_MASK, e);
        if (lane == 0 && wmax != EXP_NONE) atomicMax(block_emax ? block_emax : &ctl->emax, wmax);
    }
    const unsigned nlost = __reduce_add_sync(FULL_MASK, lost);
    const unsigned novf = __reduce_add_sync(FULL_MASK, ovf);
    if (lane == 0) {
        /* the probe pass repeats the step: only the real pass reports */
        if (nlost && DEP != DEP_PROBE) atomicAdd(&ctl->lost, (unsigned long long)nlost);
        if (novf && DEP != DEP_PROBE) atomicAdd(&ctl->overflow, (unsigned long long)novf);
    }
    amax = (A)0;
    ovf = 0;
    lost = 0;
}

}  // namespace st

#endif
