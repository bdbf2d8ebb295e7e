/*
 * st_tet.cu -- the parcel step on unstructured tetrahedral meshes with face-walk
 * relocation (the benchmark mesh: 96^3 jittered hexes split into 6 tets; no counterpart in the
 * reference, whose cuboid mesh is located by floor, A:663-697).
 *
 * Each parcel carries its owning tet.  After the drag update and the position update, a new
 * position outside the box keeps its old coordinate on that axis and mirrors the old
 * velocity component (the reference's wall rule, A:1313-1329), then a greedy walk moves from
 * the current tet across the face with the largest positive signed distance until the
 * position is inside.  The four FP64 face planes of every tet are computed once, when the
 * mesh is created (k_tet_planes), from its vertices with the vertex ids in increasing order
 * (st_create_tet sorts them and permutes the neighbours with them):
 *   face f opposite vertex f, (p, q, r) = the other vertices in increasing order,
 *   n = (q - p) x (r - p), negated if n . (v_f - p) > 0, c = n . p; s_f(x) = n . x - c;
 *   inside iff all s_f <= 0; ties between faces go to the lowest index.
 * The two tets of a shared face therefore hold the same plane bit for bit up to an exact
 * negation: a point is never outside both, and no walk bounces between two tets.  Every walk
 * step is first decided from FP32 copies of the tet's planes (64 bytes) with a proven rounding
 * bound, which settles "inside" and "leave through face f" except within about 4e-7 of the
 * plane scale of a face or of a tie; only those steps read the 128 bytes of FP64 planes.
 * The same arithmetic, without fused multiply-adds, is in the CPU oracle, so owning tets agree
 * bit for bit.  A walk that reaches a boundary face or exceeds the hop limit marks the parcel
 * as lost (its state is left unchanged and the host reports it).  Deposits use the same
 * deterministic fixed-point path as the hex kernels.
 */
#include <cstdint>
#include <cuda_runtime.h>

#include <atomic>

#include "st_device.cuh"
#include "st_ring.cuh"

namespace st {

enum { TWALK_OK = 0, TWALK_EXIT = 1, TWALK_HOPS = 2 };

/* Signed distances of x to the four face planes of tet t (planes read as 2 x 16 bytes). */
__device__ __forceinline__ void tet_signed(const TetMeshK& m, int32_t t, const double x[3],
                                           double s[4])
{
    const double2* pl = reinterpret_cast<const double2*>(m.planes + 4 * (int64_t)t);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const double2 nxy = __ldg(pl + 2 * f);
        const double2 nzc = __ldg(pl + 2 * f + 1);
        s[f] = ((nxy.x * x[0] + nxy.y * x[1]) + nzc.x * x[2]) - nzc.y;
    }
}

/* Face planes at mesh creation: face f of tet t is opposite its vertex f (vertex ids in
 * increasing order), (p, q, r) the other three in increasing order, n = (q - p) x (r - p)
 * negated if n . (v_f - p) > 0, c = n . p. */
__global__ void k_tet_planes(const double* __restrict__ verts, const int32_t* __restrict__ tets,
                             int64_t nt, double4* __restrict__ planes,
                             float4* __restrict__ planes32)
{
    const int F[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 4 * nt;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i >> 2;
        const int f = (int)(i & 3);
        const double* v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = verts + 3 * (int64_t)tets[4 * t + k];
        const double* p = v[F[f][0]];
        const double* q = v[F[f][1]];
        const double* r = v[F[f][2]];
        const double a0 = q[0] - p[0], a1 = q[1] - p[1], a2 = q[2] - p[2];
        const double b0 = r[0] - p[0], b1 = r[1] - p[1], b2 = r[2] - p[2];
        double n0 = a1 * b2 - a2 * b1;
        double n1 = a2 * b0 - a0 * b2;
        double n2 = a0 * b1 - a1 * b0;
        const double e = (n0 * (v[f][0] - p[0]) + n1 * (v[f][1] - p[1])) + n2 * (v[f][2] - p[2]);
        if (e > 0.0) { n0 = -n0; n1 = -n1; n2 = -n2; }
        const double c = (n0 * p[0] + n1 * p[1]) + n2 * p[2];
        planes[i] = make_double4(n0, n1, n2, c);
        planes32[i] = make_float4((float)n0, (float)n1, (float)n2, (float)c);
    }
}

cudaError_t launch_tet_planes(const double* verts, const int32_t* tets, int64_t nt,
                              double4* planes, float4* planes32, cudaStream_t s)
{
    if (nt == 0) return cudaSuccess;
    int64_t g = (4 * nt + 255) / 256;
    if (g > 148 * 32) g = 148 * 32;
    k_tet_planes<<<(int)g, 256, 0, s>>>(verts, tets, nt, planes, planes32);
    return cudaGetLastError();
}

/* One walk step at tet t decided from the FP32 copies of its planes (64 bytes instead of
 * the 128 bytes of FP64 ones).  Returns 1 when x is certainly inside t (every FP64 signed
 * distance negative), 2 when the FP64 test certainly leaves through face fb (its signed
 * distance positive and strictly the largest, so no tie rule applies), 0 when FP32 cannot
 * decide and the walk must evaluate the FP64 planes.  Where it decides, it decides exactly
 * as the FP64 step does.
 *
 * Bound: with u = 2^-24, n', c', x' the FP32 roundings of the FP64 plane and position, the FP32
 * evaluation s' = ((n0'x0' + n1'x1') + n2'x2') - c' (no fused multiply-adds) differs from the
 * exact s = n.x - c by at most gamma_6 S (Higham, Accuracy and Stability of Numerical
 * Algorithms, 2nd ed., sec. 3.1: six roundings on the product terms, two on c), with
 * S = sum |n_i x_i| + |c| and gamma_6 = 6u/(1 - 6u) < 3.6e-7; the FP64 evaluation differs
 * from s by at most gamma_3 S in double (< 4e-16 S).  |x_i| <= xmax inside the box, so
 * S <= (sum |n_i|) xmax + |c| <= (1 + 7u) times that sum formed in FP32 from n', c'.
 * e = 4e-7 times the FP32 sum, plus 1e-37 for rounding near the subnormal range, therefore
 * bounds |s' - s64| with a 10 % margin, which also covers the roundings of the comparisons
 * below: s' < -e gives s64 < 0, s' > e gives s64 > 0, and s'_b - s'_f > e_b + e_f gives
 * s64_f < s64_b. */
__device__ __forceinline__ int tet_step32(const TetMeshK& m, int32_t t, const float x[3], int& fb)
{
    const float4* pl = m.planes32 + 4 * (int64_t)t;
    float s[4], e[4];
    bool in = true;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
        const float4 q = __ldg(pl + f);
        s[f] = ((q.x * x[0] + q.y * x[1]) + q.z * x[2]) - q.w;
        e[f] = 4.0e-7f * (((fabsf(q.x) + fabsf(q.y)) + fabsf(q.z)) * m.xmax + fabsf(q.w)) +
               1.0e-37f;
        in = in && (s[f] < -e[f]);
    }
    if (in) return 1;
    int b = 0;
#pragma unroll
    for (int f = 1; f < 4; ++f)
        if (s[f] > s[b]) b = f;
    if (!(s[b] > e[b])) return 0;
#pragma unroll
    for (int f = 0; f < 4; ++f)
        if (f != b && !(s[b] - s[f] > e[b] + e[f])) return 0;
    fb = b;
    return 2;
}

/* Greedy walk; at most hop_limit moves (bounded loop).  Each step is decided in FP32 where
 * tet_step32 can, else from the FP64 planes; both give the FP64 walk's tets and hops. */
__device__ __forceinline__ int32_t tet_walk(const TetMeshK& m, int32_t t, const double x[3],
                                            int hop_limit, int& status, int& hops)
{
    hops = 0;
    const float x32[3] = {(float)x[0], (float)x[1], (float)x[2]};
    /* the FP32 bound holds for positions with |x_i| <= xmax (every position inside the box);
     * anything else goes straight to the FP64 test */
    const bool pre = fabs(x[0]) <= (double)m.xmax && fabs(x[1]) <= (double)m.xmax &&
                     fabs(x[2]) <= (double)m.xmax;
    for (int it = 0; it <= hop_limit; ++it) {
        int fb = 0;
        const int r = pre ? tet_step32(m, t, x32, fb) : 0;
        if (r == 1) {
            status = TWALK_OK;
            return t;
        }
        if (r == 0) {
            double s[4];
            tet_signed(m, t, x, s);
            double smax = s[0];
#pragma unroll
            for (int f = 1; f < 4; ++f)
                if (s[f] > smax) { smax = s[f]; fb = f; }
            if (!(smax > 0.0)) {
                status = TWALK_OK;
                return t;
            }
        }
        const int32_t nb = __ldg(m.nbr + 4 * (int64_t)t + fb);
        if (nb < 0) {
            status = TWALK_EXIT;
            return t;
        }
        if (hops >= hop_limit) break;
        t = nb;
        ++hops;
    }
    status = TWALK_HOPS;
    return t;
}

template <class V>
__device__ __forceinline__ int tet_find_cloud(const TetStepArgs<V>& a, int64_t tile)
{
    int lo = 0, hi = a.nclouds - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&a.clouds[mid].tile0) <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/* walk-length histogram of a block (flushed once at the end of the step kernel) */
__shared__ unsigned s_tet_hist[8];

/* One parcel through the substeps on a tet mesh (evolve_particle!, A:1271-1365, with the
 * face walk for relocation) after its state has been read: pos, vel and cell (its owning
 * tet) are updated in place unless the parcel is lost (then they are left as they were);
 * the final deposit is returned in (key, dep) for the warp reduction, intermediate deposits
 * (substeps > 1) go straight to memory.  With count_hops, walk lengths go to the block's
 * histogram s_tet_hist. */
template <class V, int DEP>
__device__ __forceinline__ void tet_parcel(const TetStepArgs<V>& a, int nsub, double pos[3],
                                           V vel[3], V d, int32_t& cell,
                                           unsigned long long* acc, double* src,
                                           const Quant& qp, AmaxT<V>& amax, unsigned& ovf,
                                           bool& lost, int32_t& key, V dep[3], bool count_hops)
{
    const PhysK<V>& ph = a.phys;
    int32_t cur = cell;
    const V mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;
    const V f = ((((V)18 * ph.mu) * a.dtV) / (ph.rho_d * (d * d))) * ph.alpha;
    constexpr bool MIX = is_mixed<double, V>;
    const V* Uc = a.U + 3 * (int64_t)cur;
    V Ur[3] = {__ldg(Uc), __ldg(Uc + 1), __ldg(Uc + 2)};
    /* deposit forms of the hex step (st_kernels.cu evolve_parcel): FP32/FP64 carry
     * state0, mixed precision carries D = state0 - v */
    V state0[3] = {vel[0], vel[1], vel[2]};
    V D[3] = {(V)0, (V)0, (V)0};
    double posNew[3] = {pos[0], pos[1], pos[2]};
    V velNew[3] = {vel[0], vel[1], vel[2]};
    int32_t tNew = cur;
    lost = false;
    for (int t = 1; t <= nsub; ++t) {
        V inc[3];
        if (ph.drag == 0) {
            if constexpr (MIX) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    inc[k] = (f * slip<MIX>(Ur[k], a.fscale, a.fscale_lo, vel[k])) /
                             ((V)1 + f);
                    velNew[k] = vel[k] + inc[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    velNew[k] = (vel[k] + f * (Ur[k] * a.fscale)) / ((V)1 + f);
            }
        } else {
            V du[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                du[k] = slip<MIX>(Ur[k], a.fscale, a.fscale_lo, vel[k]);
            V mag = st_sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2]);
            V Re = (mag * d) * ph.rnu;
            V pw;
            if (sizeof(V) == 4) pw = (V)st_pow0687f((float)Re);
            else pw = (V)st_pow0687((double)Re);
            V g = f * ((V)1 + (V)0.15 * pw);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                inc[k] = g * du[k];
                velNew[k] = vel[k] + inc[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) posNew[k] = pos[k] + (double)velNew[k] * a.dtP;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (posNew[k] < a.mesh.origin[k] || posNew[k] > a.mesh.ending[k]) {
                posNew[k] = pos[k];
                velNew[k] = -vel[k];
                if constexpr (!MIX) state0[k] -= (V)2 * vel[k];
            } else if constexpr (MIX) {
                D[k] -= inc[k];
            }
        }
        int status = TWALK_OK, hops = 0;
        tNew = tet_walk(a.mesh, tNew, posNew, a.mesh.hop_limit, status, hops);
        if (status != TWALK_OK) { lost = true; break; }
        if (count_hops) atomicAdd(&s_tet_hist[hops < 7 ? hops : 7], 1u);
        if (t != nsub && tNew != cur) {
            V di[3];
#pragma unroll
            for (int k = 0; k < 3; ++k)
                di[k] = MIX ? mB * D[k] : mB * (state0[k] - velNew[k]);
            if (DEP == DEP_PROBE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) track_max(di[k], amax);
            } else {
                deposit_direct<DEP, V>(di, (int64_t)cur, acc, src, qp, amax, ovf);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                state0[k] = velNew[k];
                D[k] = (V)0;
            }
            const V* Un = a.U + 3 * (int64_t)tNew;
            Ur[0] = __ldg(Un);
            Ur[1] = __ldg(Un + 1);
            Ur[2] = __ldg(Un + 2);
            cur = tNew;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) { vel[k] = velNew[k]; pos[k] = posNew[k]; }
    }
    if (lost) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dep[k] = MIX ? mB * D[k] : mB * (state0[k] - velNew[k]);
        pos[k] = posNew[k];
        vel[k] = velNew[k];
    }
    key = cur;
    cell = tNew;
}

/* Resident blocks of 256 threads per SM the compiler must allow: 4 (64 registers). */
#ifndef ST_TET_MIN_BLOCKS
#define ST_TET_MIN_BLOCKS 4
#endif
template <class V>
struct TetMinBlocks {
    static constexpr int value = ST_TET_MIN_BLOCKS;
};

template <class V, int DEP, bool ONE>
__global__ void __launch_bounds__(256, TetMinBlocks<V>::value) k_step_tet(const TetStepArgs<V> a)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr bool DET = (DEP == DEP_DET1 || DEP == DEP_DET2);
    const PhysK<V>& ph = a.phys;
    int cur_cloud = -1;
    Quant qp = {0.0, 0.0, 0.0f, 0.0f, 0, false};
    AmaxT<V> amax = (V)0;
    unsigned ovf = 0, nlost = 0;
    const int nsub = ONE ? 1 : ph.nsub;
    const bool count_hops = a.hop_hist != nullptr && DEP != DEP_PROBE;
    if (threadIdx.x < 8) s_tet_hist[threadIdx.x] = 0;
    __syncthreads();

    for (int64_t tile = warp0; tile < a.total_tiles; tile += nwarps) {
        const int c = (a.nclouds == 1) ? 0 : tet_find_cloud(a, tile);
        if (c != cur_cloud) {
            if (cur_cloud >= 0) flush_ctl<DEP>(a.ctl + cur_cloud, lane, amax, ovf, nlost);
            cur_cloud = c;
            if (DET) qp = make_quant(a.ctl[c].L, a.ctl[c].H + QUANT_GROWTH_BITS);
        }
        const CloudK<double, V>* cl = a.clouds + c;
        const int64_t n = __ldg(&cl->n);
        unsigned long long* const acc = DET ? cl->acc : nullptr;
        double* const src = (DEP == DEP_ATOMIC) ? cl->src : nullptr;
        for (int sl = 0; sl < WARP_TILE / 32; ++sl) {
        const int64_t i = (tile - __ldg(&cl->tile0)) * WARP_TILE + 32 * sl + lane;
        int32_t key = -1;
        V dep[3] = {(V)0, (V)0, (V)0};
        if (i < n) {
            double pos[3] = {ld_stream(cl->x + i), ld_stream(cl->y + i), ld_stream(cl->z + i)};
            V vel[3] = {ld_stream(cl->u + i), ld_stream(cl->v + i), ld_stream(cl->w + i)};
            const V d = ld_stream(cl->d + i) * ph.dscale;
            int32_t cell = ld_stream(cl->cell + i);
            /* the first walk step reads this tet's FP32 planes: start that line towards L1
             * now, alongside the cell-velocity gather */
            asm volatile("prefetch.global.L1 [%0];" ::"l"(a.mesh.planes32 + 4 * (int64_t)cell));
            bool lost = false;
            tet_parcel<V, DEP>(a, nsub, pos, vel, d, cell, acc, src, qp, amax, ovf, lost, key,
                               dep, count_hops);
            if (lost) {
                ++nlost;
                key = -1;
            } else if (DEP != DEP_PROBE) {
                st_stream(cl->x + i, pos[0]);
                st_stream(cl->y + i, pos[1]);
                st_stream(cl->z + i, pos[2]);
                st_stream(cl->u + i, vel[0]);
                st_stream(cl->v + i, vel[1]);
                st_stream(cl->w + i, vel[2]);
                st_stream(cl->cell + i, cell);
            }
        }
        deposit_warp<DEP, V>(key, dep, acc, src, qp, lane, amax, ovf);
        }
    }
    if (cur_cloud >= 0) flush_ctl<DEP>(a.ctl + cur_cloud, lane, amax, ovf, nlost);
    __syncthreads();
    if (count_hops && threadIdx.x < 8 && s_tet_hist[threadIdx.x])
        atomicAdd(a.hop_hist + threadIdx.x, (unsigned long long)s_tet_hist[threadIdx.x]);
}

/* ------------------------------------------------------------------------------------ */
/* the tet step of one cloud on the shared-memory ring                                  */
/* ------------------------------------------------------------------------------------ */

/* 992-parcel tiles, 31 consumer warps with one slice each (32 warps at 64 registers: the
 * walk's chains of dependent gathers need many warps in flight) */
using TetShape = RingShape<992, 31>;

/* The consumer work of the tet ring: each warp's slices of 32 parcels through
 * tet_parcel, the new state written back into the tile, deposits reduced per slice. */
template <class V, int DEP, bool ONE>
struct TetRing {
    const TetStepArgs<V>& a;
    unsigned long long* acc;
    double* src;
    const Quant& qp;
    int lane;
    bool count_hops;
    AmaxT<V>& amax;
    unsigned& ovf;
    unsigned& nlost;
    template <bool GLOBAL>
    __device__ __forceinline__ void run(const RingArrays<double, V>& r, int j0, int64_t nvalid)
    {
        const int nsub = ONE ? 1 : a.phys.nsub;
#pragma unroll
        for (int sl = 0; sl < TetShape::SPW; ++sl) {
            const int j = j0 + 32 * sl;
            int32_t key = -1;
            V dep[3] = {(V)0, (V)0, (V)0};
            if (!GLOBAL || j < nvalid) {
                double pos[3] = {ring_ld<GLOBAL>(r.x + j), ring_ld<GLOBAL>(r.y + j),
                                 ring_ld<GLOBAL>(r.z + j)};
                V vel[3] = {ring_ld<GLOBAL>(r.u + j), ring_ld<GLOBAL>(r.v + j),
                            ring_ld<GLOBAL>(r.w + j)};
                const V d = ring_ld<GLOBAL>(r.d + j) * a.phys.dscale;
                int32_t cell = ring_ld<GLOBAL>(r.cell + j);
                bool lost = false;
                tet_parcel<V, DEP>(a, nsub, pos, vel, d, cell, acc, src, qp, amax, ovf, lost,
                                   key, dep, count_hops);
                if (lost) {
                    ++nlost;
                    key = -1;
                } else {
                    ring_st<GLOBAL>(r.x + j, pos[0]);
                    ring_st<GLOBAL>(r.y + j, pos[1]);
                    ring_st<GLOBAL>(r.z + j, pos[2]);
                    ring_st<GLOBAL>(r.u + j, vel[0]);
                    ring_st<GLOBAL>(r.v + j, vel[1]);
                    ring_st<GLOBAL>(r.w + j, vel[2]);
                    ring_st<GLOBAL>(r.cell + j, cell);
                }
            }
            deposit_warp<DEP, V>(key, dep, acc, src, qp, lane, amax, ovf);
        }
    }
};

template <class V, int DEP, bool ONE>
__global__ void __launch_bounds__(TetShape::THREADS, 1) k_step_tet_ring(const TetStepArgs<V> a)
{
    constexpr bool DET = (DEP == DEP_DET1 || DEP == DEP_DET2);
    Quant qp = {0.0, 0.0, 0.0f, 0.0f, 0, false};
    if (DET) qp = make_quant(a.ctl[0].L, a.ctl[0].H + QUANT_GROWTH_BITS);
    AmaxT<V> amax = (V)0;
    unsigned ovf = 0, nlost = 0;
    const int lane = threadIdx.x & 31;
    const bool count_hops = a.hop_hist != nullptr;
    if (threadIdx.x < 8) s_tet_hist[threadIdx.x] = 0;   /* ring_block synchronises */
    ring_emax_init();
    TetRing<V, DEP, ONE> step{a, DET ? a.one.acc : nullptr,
                              DEP == DEP_ATOMIC ? a.one.src : nullptr, qp, lane, count_hops,
                              amax, ovf, nlost};
    if (!ring_block<TetShape, double, V, true>(a.one, a.ctl, step, a.wait_cycles)) return;
    flush_ctl<DEP>(a.ctl, lane, amax, ovf, nlost, DEP != DEP_ATOMIC ? &s_ring_emax : nullptr);
    ring_consumers_sync<TetShape>();
    if (count_hops && threadIdx.x < 8 && s_tet_hist[threadIdx.x])
        atomicAdd(a.hop_hist + threadIdx.x, (unsigned long long)s_tet_hist[threadIdx.x]);
    /* one device-scope atomic per block on the cloud's exponent word (see ring_emax_flush) */
    if (DEP != DEP_ATOMIC && threadIdx.x == 0 && s_ring_emax != EXP_NONE)
        atomicMax(&a.ctl->emax, s_ring_emax);
}

template <class V, int DEP, bool ONE>
static cudaError_t tet_ring_attr()
{
    static std::atomic<unsigned long long> ready{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ULL << (dev & 63);
    if (ready.load() & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(k_step_tet_ring<V, DEP, ONE>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)RingGeom<TetShape, double, V, true>::SMEM);
    if (e == cudaSuccess) ready.fetch_or(bit);
    return e;
}

template <class V, int DEP, bool ONE>
static cudaError_t launch_tet_ring_t(const TetStepArgs<V>& a, int nsm, cudaStream_t s)
{
    cudaError_t e = tet_ring_attr<V, DEP, ONE>();
    if (e != cudaSuccess) return e;
    const int64_t nfull = a.one.n / TetShape::BT;
    int64_t grid = nfull < nsm ? nfull : nsm;
    if (grid < 1) grid = 1;
    k_step_tet_ring<V, DEP, ONE>
        <<<(int)grid, TetShape::THREADS, RingGeom<TetShape, double, V, true>::SMEM, s>>>(a);
    return cudaGetLastError();
}

template <class V>
bool tet_ring_eligible(const TetStepArgs<V>& a, int dep)
{
    if (a.nclouds != 1 || a.one.n <= 0 || !a.one.cell) return false;
    if (dep != DEP_DET1 && dep != DEP_DET2 && dep != DEP_ATOMIC) return false;
    const void* p[8] = {a.one.x, a.one.y, a.one.z, a.one.u, a.one.v, a.one.w, a.one.d, a.one.cell};
    for (const void* q : p)
        if (reinterpret_cast<uintptr_t>(q) % 16) return false;
    return true;
}

template <class V>
cudaError_t launch_step_tet_ring(const TetStepArgs<V>& a, int dep, int nsm, cudaStream_t s)
{
    const bool one = a.phys.nsub == 1;
    switch (dep) {
    case DEP_DET1: return one ? launch_tet_ring_t<V, DEP_DET1, true>(a, nsm, s)
                              : launch_tet_ring_t<V, DEP_DET1, false>(a, nsm, s);
    case DEP_DET2: return one ? launch_tet_ring_t<V, DEP_DET2, true>(a, nsm, s)
                              : launch_tet_ring_t<V, DEP_DET2, false>(a, nsm, s);
    case DEP_ATOMIC: return one ? launch_tet_ring_t<V, DEP_ATOMIC, true>(a, nsm, s)
                                : launch_tet_ring_t<V, DEP_ATOMIC, false>(a, nsm, s);
    default: return cudaErrorInvalidValue;
    }
}

/* Makes every tet ring kernel instance of a precision launchable on the current device
 * (called when a tet handle is created, outside any stream capture). */
template <class V>
cudaError_t tet_ring_prepare()
{
    const cudaError_t r[6] = {tet_ring_attr<V, DEP_DET1, true>(), tet_ring_attr<V, DEP_DET1, false>(),
                              tet_ring_attr<V, DEP_DET2, true>(), tet_ring_attr<V, DEP_DET2, false>(),
                              tet_ring_attr<V, DEP_ATOMIC, true>(),
                              tet_ring_attr<V, DEP_ATOMIC, false>()};
    for (cudaError_t e : r)
        if (e != cudaSuccess) return e;
    return cudaSuccess;
}

template bool tet_ring_eligible<float>(const TetStepArgs<float>&, int);
template bool tet_ring_eligible<double>(const TetStepArgs<double>&, int);
template cudaError_t launch_step_tet_ring<float>(const TetStepArgs<float>&, int, int, cudaStream_t);
template cudaError_t launch_step_tet_ring<double>(const TetStepArgs<double>&, int, int, cudaStream_t);
template cudaError_t tet_ring_prepare<float>();
template cudaError_t tet_ring_prepare<double>();

template <class V, bool ONE>
static cudaError_t launch_step_tet_t(const TetStepArgs<V>& a, int dep, int grid, int block,
                                     cudaStream_t s)
{
    switch (dep) {
    case DEP_DET1: k_step_tet<V, DEP_DET1, ONE><<<grid, block, 0, s>>>(a); break;
    case DEP_DET2: k_step_tet<V, DEP_DET2, ONE><<<grid, block, 0, s>>>(a); break;
    case DEP_ATOMIC: k_step_tet<V, DEP_ATOMIC, ONE><<<grid, block, 0, s>>>(a); break;
    case DEP_PROBE: k_step_tet<V, DEP_PROBE, ONE><<<grid, block, 0, s>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class V>
cudaError_t launch_step_tet(const TetStepArgs<V>& a, int dep, int grid, int block, cudaStream_t s)
{
    return a.phys.nsub == 1 ? launch_step_tet_t<V, true>(a, dep, grid, block, s)
                            : launch_step_tet_t<V, false>(a, dep, grid, block, s);
}

template <class V, bool ONE>
static int tet_max_active_t(int dep, int block)
{
    int nb = 0;
    cudaError_t e = cudaErrorInvalidValue;
    switch (dep) {
    case DEP_DET1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step_tet<V, DEP_DET1, ONE>, block, 0); break;
    case DEP_DET2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step_tet<V, DEP_DET2, ONE>, block, 0); break;
    case DEP_ATOMIC: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step_tet<V, DEP_ATOMIC, ONE>, block, 0); break;
    case DEP_PROBE: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step_tet<V, DEP_PROBE, ONE>, block, 0); break;
    default: break;
    }
    return e == cudaSuccess ? nb : 0;
}

template <class V>
int step_tet_max_active_blocks(int dep, int block)
{
    const int x = tet_max_active_t<V, true>(dep, block);
    const int y = tet_max_active_t<V, false>(dep, block);
    return x < y ? x : y;
}

__global__ void k_tet_locate(const TetMeshK m, const double* __restrict__ x,
                             const double* __restrict__ y, const double* __restrict__ z,
                             const int32_t* __restrict__ hint, int64_t n,
                             int32_t* __restrict__ cells, unsigned long long* outside)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p[3] = {x[i], y[i], z[i]};
        int32_t h = hint[i];
        int status = TWALK_EXIT, hops = 0;
        int32_t t = -1;
        if (h >= 0 && h < m.nt) t = tet_walk(m, h, p, m.hop_limit, status, hops);
        const bool ok = status == TWALK_OK;
        cells[i] = ok ? t : -1;
        if (!ok) atomicAdd(outside, 1ULL);
    }
}

cudaError_t launch_tet_locate(const TetMeshK& m, const double* x, const double* y,
                              const double* z, const int32_t* hint, int64_t n, int32_t* cells,
                              unsigned long long* outside, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_tet_locate<<<(int)g, 256, 0, s>>>(m, x, y, z, hint, n, cells, outside);
    return cudaGetLastError();
}

template cudaError_t launch_step_tet<float>(const TetStepArgs<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_step_tet<double>(const TetStepArgs<double>&, int, int, int, cudaStream_t);
template int step_tet_max_active_blocks<float>(int, int);
template int step_tet_max_active_blocks<double>(int, int);

}  // namespace st
