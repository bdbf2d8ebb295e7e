/*
 * st_adjoint.cu -- adjoint of the parcel step for the time-averaged source (no counterpart
 * in the reference, which has no adjoint).
 *
 * Objective-side contract (the pull-back of y = Sbar = (1/T) sum_n S_n): given the cotangent
 * ybar = dJ/dSbar per cell, return dJ/dalpha (drag multiplier), dJ/ds (diameter scale) and
 * dJ/dv0 per parcel, with cell ownership and wall-bounce decisions frozen at the forward
 * pass.  Schiller-Naumann drag, one substep.  Mathematics (forward and reverse step):
 *   u = U[c_n] fs_n, d_e = s d, f = 18 mu dt alpha / (rho_d d_e^2), du = u - v,
 *   Re = |du| d_e rnu, P = Re^0.687, g = f (1 + 0.15 P)
 *   v'_k = v_k + g du_k  (-v_k if bounced),  D_k = m (v_k - v'_k)  (0 if bounced)
 *   w_k = a_k - m G_k (not bounced), Sw = sum w_k du_k, gamma = 0.10305 f P / |du|^2
 *   a_j <- [not bounced]((1-g) w_j + m G_j) - [bounced] a_j - gamma du_j Sw
 *   dJ/dalpha += Sw g / alpha,  dJ/ds += Sw (-2g + 0.10305 f P)/s + (3/s) sum G_k D_k
 * with G = ybar / T.
 *
 * Kernels: k_adj_forward runs all T steps of a parcel in registers (the mean-source
 * objective only needs the sum over steps), writes checkpoints of (x, v) every C steps and
 * deposits every step into one fixed-point accumulator with a constant scale.  k_adj_reverse
 * handles one checkpoint segment: it recomputes the C forward steps from the checkpoint,
 * recording (v_n, cell, bounce flags), then runs the reverse steps back to the checkpoint,
 * keeping the parcel's cotangent and its FP64 parameter partials in registers.  Parameter
 * partials are reduced per block in shared memory in a fixed order and summed on the host in
 * block order, so the gradient is reproducible.
 */
#include <cstdint>
#include <cuda_runtime.h>

#include "st_device.cuh"

namespace st {

#define ADJ_FULL 0xffffffffu

__device__ __forceinline__ float adj_sqrt(float v) { return __fsqrt_rn(v); }
__device__ __forceinline__ double adj_sqrt(double v) { return __dsqrt_rn(v); }
__device__ __forceinline__ float adj_floor(float v) { return floorf(v); }
__device__ __forceinline__ double adj_floor(double v) { return floor(v); }

template <class P>
__device__ __forceinline__ int32_t adj_floor_label(P v, bool& bad)
{
    P f = adj_floor(v);
    if (!(f >= (P)-2147483648.0 && f < (P)2147483648.0)) {
        bad = true;
        return 0;
    }
    return (int32_t)f;
}

/* locate (A:663-697, one partition): 1-based posI and partition index */
template <class P>
__device__ __forceinline__ void adj_locate(const MeshK<P>& m, const P x[3], int32_t ijk[3],
                                           int32_t& posI, int32_t& part, bool& bad)
{
    for (int a = 0; a < 3; ++a) ijk[a] = adj_floor_label((x[a] - m.origin[a]) * m.rD[a], bad);
    int32_t q[3], r[3];
    for (int a = 0; a < 3; ++a) {
        if ((uint32_t)ijk[a] < (uint32_t)m.N[a]) {
            q[a] = 0;
            r[a] = ijk[a];
        } else {
            q[a] = ijk[a] / m.N[a];
            r[a] = ijk[a] - q[a] * m.N[a];
        }
    }
    part = abs(q[2]) + abs(q[1]) + abs(q[0]) + 1;
    posI = abs(r[2]) * m.NxNy + abs(r[1]) * m.N[0] + abs(r[0]) + 1;
}

template <class V>
struct AdjLocal {
    V mB, f, g, pw, mag2;
    V du[3];
    V dep[3];
};

/* One forward step (evolve_particle!, nSteps = 1).  Returns false if the parcel is lost. */
template <class P, class V>
__device__ __forceinline__ bool adj_step(const AdjArgs<P, V>& a, P pos[3], V vel[3], V d,
                                         V fs, V fs_lo, int32_t& cell, uint8_t& bounce,
                                         AdjLocal<V>& o)
{
    constexpr bool MIX = is_mixed<P, V>;
    const MeshK<P>& m = a.mesh;
    const PhysK<V>& ph = a.phys;
    bool bad = false;
    int32_t ijk[3], posI, part;
    adj_locate(m, pos, ijk, posI, part, bad);
    if (bad || part != 1) return false;
    o.mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;
    const V* Uc = a.U + 3 * (int64_t)(posI - 1);
    o.f = ((((V)18 * ph.mu) * a.dtV) / (ph.rho_d * (d * d))) * ph.alpha;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.du[k] = slip<MIX>(__ldg(Uc + k), fs, fs_lo, vel[k]);
    o.mag2 = (o.du[0] * o.du[0] + o.du[1] * o.du[1]) + o.du[2] * o.du[2];
    const V mag = adj_sqrt(o.mag2);
    const V Re = (mag * d) * ph.rnu;
    if (sizeof(V) == 4) o.pw = (V)st_pow0687f((float)Re);
    else o.pw = (V)st_pow0687((double)Re);
    o.g = o.f * ((V)1 + (V)0.15 * o.pw);
    P posNew[3];
    V velNew[3], inc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        inc[k] = o.g * o.du[k];
        velNew[k] = vel[k] + inc[k];
        posNew[k] = pos[k] + (P)velNew[k] * a.dtP;
    }
    uint8_t b = 0;
    int32_t nijk[3], nposI, npart;
    adj_locate(m, posNew, nijk, nposI, npart, bad);
    if (bad) return false;
    if (nposI != posI || npart != 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (nijk[k] < 0 || nijk[k] >= m.N[k]) b |= (uint8_t)(1 << k);
    }
    V state0[3] = {vel[0], vel[1], vel[2]};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (b & (1 << k)) {
            posNew[k] = pos[k];
            velNew[k] = -vel[k];
            state0[k] -= (V)2 * vel[k];
        }
    }
    /* deposit forms of the step kernel (st_kernels.cu evolve_one): mixed precision deposits
     * -m/rho_c times the velocity increment, zero on a bounced component */
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if constexpr (MIX) o.dep[k] = o.mB * ((b & (1 << k)) ? (V)0 : -inc[k]);
        else o.dep[k] = o.mB * (state0[k] - velNew[k]);
        pos[k] = posNew[k];
        vel[k] = velNew[k];
    }
    cell = posI - 1;
    bounce = b;
    return true;
}

/* Reverse step: vel = velocity at the start of the step, a = cotangent after the step (in)
 * and before it (out). */
template <class P, class V>
__device__ __forceinline__ void adj_reverse(const AdjArgs<P, V>& a, const V vel[3], V d, V fs,
                                            V fs_lo,
                                            int32_t cell, uint8_t b, V av[3], double& dalpha,
                                            double& dscale)
{
    constexpr bool MIX = is_mixed<P, V>;
    const PhysK<V>& ph = a.phys;
    AdjLocal<V> o;
    o.mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;
    const V* Uc = a.U + 3 * (int64_t)cell;
    o.f = ((((V)18 * ph.mu) * a.dtV) / (ph.rho_d * (d * d))) * ph.alpha;
#pragma unroll
    for (int k = 0; k < 3; ++k) o.du[k] = slip<MIX>(__ldg(Uc + k), fs, fs_lo, vel[k]);
    o.mag2 = (o.du[0] * o.du[0] + o.du[1] * o.du[1]) + o.du[2] * o.du[2];
    const V mag = adj_sqrt(o.mag2);
    const V Re = (mag * d) * ph.rnu;
    if (sizeof(V) == 4) o.pw = (V)st_pow0687f((float)Re);
    else o.pw = (V)st_pow0687((double)Re);
    o.g = o.f * ((V)1 + (V)0.15 * o.pw);
    V velNew[3], state0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const V inc = o.g * o.du[k];
        velNew[k] = vel[k] + inc;
        state0[k] = vel[k];
        if (b & (1 << k)) {
            velNew[k] = -vel[k];
            state0[k] -= (V)2 * vel[k];
        }
        if constexpr (MIX) o.dep[k] = o.mB * ((b & (1 << k)) ? (V)0 : -inc);
        else o.dep[k] = o.mB * (state0[k] - velNew[k]);
    }
    const double* Gd = a.G + 3 * (int64_t)cell;
    const V G[3] = {(V)__ldg(Gd), (V)__ldg(Gd + 1), (V)__ldg(Gd + 2)};
    V w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = (b & (1 << k)) ? (V)0 : av[k] - o.mB * G[k];
    const V Sw = (w[0] * o.du[0] + w[1] * o.du[1]) + w[2] * o.du[2];
    const V gamma = o.mag2 > (V)0 ? (((V)0.10305 * o.f) * o.pw) / o.mag2 : (V)0;
    V an[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const V t = (b & (1 << j)) ? -av[j] : ((V)1 - o.g) * w[j] + o.mB * G[j];
        an[j] = t - (gamma * o.du[j]) * Sw;
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) av[j] = an[j];
    dalpha += (double)(Sw * (o.g / ph.alpha));
    const V GD = (G[0] * o.dep[0] + G[1] * o.dep[1]) + G[2] * o.dep[2];
    dscale += (double)((Sw * ((V)-2 * o.g + ((V)0.10305 * o.f) * o.pw)) / ph.dscale +
                       ((V)3 / ph.dscale) * GD);
}

__device__ __forceinline__ float adj_abs(float v) { return fabsf(v); }
__device__ __forceinline__ double adj_abs(double v) { return fabs(v); }

/* MODE 0: probe (first step, largest |deposit| only).  MODE 1: all T steps with
 * checkpoints and the fixed-point mean-source accumulation. */
template <class P, class V, int MODE>
__global__ void __launch_bounds__(256) k_adj_forward(const AdjArgs<P, V> a)
{
    const int lane = threadIdx.x & 31;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = i < a.n;
    P pos[3];
    V vel[3], d = (V)0;
    if (active) {
        pos[0] = a.x[i]; pos[1] = a.y[i]; pos[2] = a.z[i];
        vel[0] = a.u[i]; vel[1] = a.v[i]; vel[2] = a.w[i];
        d = a.d[i] * a.phys.dscale;
    }
    bool alive = active;
    double amax = 0.0;
    unsigned lost = 0, ovf = 0;
    const int nsteps = MODE == 0 ? 1 : a.T;
    /* fixed-point parameters of the mean accumulator (constant over the run) */
    const int L = a.ctl->L;
    const int cap = a.ctl->H + QUANT_GROWTH_BITS;
    const double scale = (-L >= -1022 && -L <= 1023) ? st_pow2i(-L) : 0.0;
    for (int n = 0; n < nsteps; ++n) {
        if (MODE == 1 && (n % a.C) == 0 && active) {
            const int64_t k = n / a.C;
            P* cx = a.ck_x + k * 3 * a.n;
            V* cv = a.ck_v + k * 3 * a.n;
            cx[i] = pos[0]; cx[a.n + i] = pos[1]; cx[2 * a.n + i] = pos[2];
            cv[i] = vel[0]; cv[a.n + i] = vel[1]; cv[2 * a.n + i] = vel[2];
        }
        int32_t key = -1;
        V dep[3] = {(V)0, (V)0, (V)0};
        if (alive) {
            int32_t cell;
            uint8_t b;
            AdjLocal<V> o;
            if (adj_step<P, V>(a, pos, vel, d, a.fs[n], a.fs_lo[n], cell, b, o)) {
                key = cell;
#pragma unroll
                for (int k = 0; k < 3; ++k) dep[k] = o.dep[k];
            } else {
                alive = false;
                ++lost;
            }
        }
        if (MODE == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double v = fabs((double)dep[k]);
                if (v < __longlong_as_double(0x7ff0000000000000LL)) amax = fmax(amax, v);
            }
            continue;
        }
        /* one limb (V = float) or two (V = double), exact integer sums */
        long long q[3] = {0, 0, 0};
        if (key >= 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double dv = (double)dep[k];
                if (dv == 0.0) continue;
                const double av = fabs(dv);
                if (!(av < __longlong_as_double(0x7ff0000000000000LL))) { ++ovf; continue; }
                int e;
                {
                    uint64_t bb = (uint64_t)__double_as_longlong(av);
                    int be = (int)(bb >> 52);
                    if (be == 0) {
                        double sc = av * 18014398509481984.0;
                        be = (int)(((uint64_t)__double_as_longlong(sc)) >> 52) - 54;
                    }
                    e = be - 1022;
                }
                if (e - L > cap) { ++ovf; continue; }
                const double x = scale != 0.0 ? dv * scale
                                              : (dv * st_pow2i(-L / 2)) * st_pow2i(-L - (-L / 2));
                q[k] = __double2ll_rn(x);
            }
        }
        /* runs of equal cells among the warp's lanes: one atomic per run and component */
        const int prev = __shfl_up_sync(ADJ_FULL, key, 1);
        const bool head = (lane == 0) || (prev != key);
        const unsigned heads = __ballot_sync(ADJ_FULL, head);
        const int segstart = 31 - __clz(heads & (ADJ_FULL >> (31 - lane)));
        const bool tail = (lane == 31) || ((heads >> (lane + 1)) & 1u);
        if (a.limbs == 1) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                long long vv = q[k];
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    long long t = __shfl_up_sync(ADJ_FULL, vv, off);
                    if (lane - off >= segstart) vv += t;
                }
                if (tail && key >= 0 && vv) atomicAdd(a.acc + 3 * (int64_t)key + k,
                                                       (unsigned long long)vv);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                long long hv = q[k] >> 32;
                unsigned long long lv = (unsigned long long)q[k] & 0xffffffffULL;
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    long long t = __shfl_up_sync(ADJ_FULL, hv, off);
                    unsigned long long u = __shfl_up_sync(ADJ_FULL, lv, off);
                    if (lane - off >= segstart) { hv += t; lv += u; }
                }
                if (tail && key >= 0) {
                    if (hv) atomicAdd(a.acc + 2 * (3 * (int64_t)key + k), (unsigned long long)hv);
                    if (lv) atomicAdd(a.acc + 2 * (3 * (int64_t)key + k) + 1, lv);
                }
            }
        }
    }
    if (MODE == 0) {
        int e = EXP_NONE;
        if (amax > 0.0) {  /* frexp exponent of amax */
            int be = (int)(((uint64_t)__double_as_longlong(amax)) >> 52);
            if (be == 0)
                be = (int)(((uint64_t)__double_as_longlong(amax * 18014398509481984.0)) >> 52) - 54;
            e = be - 1022;
        }
        const int wmax = __reduce_max_sync(ADJ_FULL, e);
        if (lane == 0 && wmax != EXP_NONE) atomicMax(&a.ctl->emax, wmax);
    }
    const unsigned nl = __reduce_add_sync(ADJ_FULL, lost);
    const unsigned no = __reduce_add_sync(ADJ_FULL, ovf);
    if (lane == 0) {
        if (nl) atomicAdd(&a.ctl->lost, (unsigned long long)nl);
        if (no) atomicAdd(&a.ctl->overflow, (unsigned long long)no);
    }
}

/* One checkpoint segment [k C, k C + len) in reverse. */
template <class P, class V>
__global__ void __launch_bounds__(256) k_adj_reverse(const AdjArgs<P, V> a, int seg, int len)
{
    __shared__ double red[2][256];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double dalpha = 0.0, dscale = 0.0;
    if (i < a.n) {
        const P* cx = a.ck_x + (int64_t)seg * 3 * a.n;
        const V* cv = a.ck_v + (int64_t)seg * 3 * a.n;
        P pos[3] = {cx[i], cx[a.n + i], cx[2 * a.n + i]};
        V vel[3] = {cv[i], cv[a.n + i], cv[2 * a.n + i]};
        const V d = a.d[i] * a.phys.dscale;
        const int n0 = seg * a.C;
        bool ok = true;
        for (int t = 0; t < len; ++t) {           /* recompute, recording the forward */
            V* rv = a.rec_v + (int64_t)t * 3 * a.n;
            rv[i] = vel[0]; rv[a.n + i] = vel[1]; rv[2 * a.n + i] = vel[2];
            int32_t cell = -1;
            uint8_t b = 0;
            AdjLocal<V> o;
            if (ok && !adj_step<P, V>(a, pos, vel, d, a.fs[n0 + t], a.fs_lo[n0 + t], cell, b,
                                      o))
                ok = false;
            a.rec_c[(int64_t)t * a.n + i] = ok ? cell : -1;
            a.rec_b[(int64_t)t * a.n + i] = b;
        }
        V av[3] = {a.adj_v[i], a.adj_v[a.n + i], a.adj_v[2 * a.n + i]};
        for (int t = len - 1; t >= 0; --t) {      /* reverse */
            const int32_t cell = a.rec_c[(int64_t)t * a.n + i];
            if (cell < 0) continue;
            const V* rv = a.rec_v + (int64_t)t * 3 * a.n;
            const V vn[3] = {rv[i], rv[a.n + i], rv[2 * a.n + i]};
            adj_reverse<P, V>(a, vn, d, a.fs[n0 + t], a.fs_lo[n0 + t], cell,
                              a.rec_b[(int64_t)t * a.n + i], av, dalpha, dscale);
        }
        a.adj_v[i] = av[0]; a.adj_v[a.n + i] = av[1]; a.adj_v[2 * a.n + i] = av[2];
    }
    red[0][threadIdx.x] = dalpha;
    red[1][threadIdx.x] = dscale;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.partials[2 * ((int64_t)seg * gridDim.x + blockIdx.x)] = red[0][0];
        a.partials[2 * ((int64_t)seg * gridDim.x + blockIdx.x) + 1] = red[1][0];
    }
}

/* Mean source (1/T) * fixed point -> FP64, into `mean` [ncomp]. */
__global__ void k_adj_mean(const unsigned long long* __restrict__ acc, const CloudCtl* ctl,
                           int limbs, double T, double* __restrict__ mean, int64_t ncomp)
{
    const int L = ctl->L;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ncomp;
         j += (int64_t)gridDim.x * blockDim.x) {
        double v;
        if (limbs == 1) {
            v = (double)(long long)acc[j];
        } else {
            long long hi = (long long)acc[2 * j];
            unsigned long long lo = acc[2 * j + 1];
            hi += (long long)(lo >> 32);
            lo &= 0xffffffffULL;
            v = (double)hi * 4294967296.0 + (double)lo;
        }
        const int k1 = L / 2, k2 = L - L / 2;
        mean[j] = ((v * st_pow2i(k1)) * st_pow2i(k2)) / T;
    }
}

/* After the probe: a constant scale for the whole run. */
__global__ void k_adj_scale(CloudCtl* ctl)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const int em = ctl->emax;
        ctl->L = (em == EXP_NONE) ? -ctl->H : em - ctl->H;
        ctl->emax = EXP_NONE;
    }
}

template <class P, class V>
cudaError_t launch_adj_forward(const AdjArgs<P, V>& a, bool probe, cudaStream_t s)
{
    const int grid = (int)((a.n + 255) / 256);
    if (grid == 0) return cudaSuccess;
    if (probe) k_adj_forward<P, V, 0><<<grid, 256, 0, s>>>(a);
    else k_adj_forward<P, V, 1><<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

template <class P, class V>
cudaError_t launch_adj_reverse(const AdjArgs<P, V>& a, int seg, int len, int grid,
                               cudaStream_t s)
{
    if (grid == 0) return cudaSuccess;
    k_adj_reverse<P, V><<<grid, 256, 0, s>>>(a, seg, len);
    return cudaGetLastError();
}

cudaError_t launch_adj_scale(CloudCtl* ctl, cudaStream_t s)
{
    k_adj_scale<<<1, 32, 0, s>>>(ctl);
    return cudaGetLastError();
}

cudaError_t launch_adj_mean(const unsigned long long* acc, const CloudCtl* ctl, int limbs,
                            int T, double* mean, int64_t ncomp, cudaStream_t s)
{
    int grid = (int)((ncomp + 255) / 256 < 148 * 8 ? (ncomp + 255) / 256 : 148 * 8);
    if (grid < 1) grid = 1;
    k_adj_mean<<<grid, 256, 0, s>>>(acc, ctl, limbs, (double)T, mean, ncomp);
    return cudaGetLastError();
}

template cudaError_t launch_adj_forward<double, float>(const AdjArgs<double, float>&, bool, cudaStream_t);
template cudaError_t launch_adj_forward<double, double>(const AdjArgs<double, double>&, bool, cudaStream_t);
template cudaError_t launch_adj_reverse<double, float>(const AdjArgs<double, float>&, int, int, int, cudaStream_t);
template cudaError_t launch_adj_reverse<double, double>(const AdjArgs<double, double>&, int, int, int, cudaStream_t);

}  // namespace st
