/*
 * st_step.cuh -- one parcel through one call of the step on the uniform hex mesh: locate
 * (A:663-697) and evolve_particle! (A:1271-1365) in the precision modes of the library.
 * Shared by the warp-tile step kernel (st_kernels.cu) and the shared-memory ring kernel
 * (st_ring.cu).
 *
 * Reference: A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 */
#ifndef ST_STEP_CUH
#define ST_STEP_CUH

#include "st_device.cuh"

namespace st {

/* ------------------------------------------------------------------------------------ */
/* relocation                                                                           */
/* ------------------------------------------------------------------------------------ */

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
    if ((uint32_t)r.I < (uint32_t)m.N[0] && (uint32_t)r.J < (uint32_t)m.N[1] &&
        (uint32_t)r.K < (uint32_t)m.N[2]) {  /* inside: divrem is (0, i) on every axis */
        r.part = 1;
        r.posI = r.K * m.NxNy + r.J * m.N[0] + r.I + 1;
        return r;
    }
    int32_t iP, iL, jP, jL, kP, kL;
    divrem_label(r.I, m.N[0], iP, iL);
    divrem_label(r.J, m.N[1], jP, jL);
    divrem_label(r.K, m.N[2], kP, kL);
    r.part = abs(kP) + abs(jP) + abs(iP) + 1;
    r.posI = abs(kL) * m.NxNy + abs(jL) * m.N[0] + abs(iL) + 1;
    return r;
}

/* One parcel through all substeps (A:1271-1365) after its start cell has been located and
 * its raw cell velocity Ur gathered.  pos/vel are updated in place; the final deposit is
 * returned in (key, dep) for the warp-level reduction; intermediate deposits on cell change
 * (A:1342-1348, only with substeps > 1) go straight to memory.
 *
 * FP32 and FP64 follow the reference's form: state0 = v at the last deposit, the deposit is
 * m/rho_c (state0 - v'), and a wall bounce sets v'_c = -v_c with state0_c -= 2 v_c.  Mixed
 * precision carries D = state0 - v instead: each substep subtracts its velocity increment
 * (a bounced component keeps its D, the bounce moves no momentum to the fluid) and the deposit
 * is m/rho_c D.  In exact arithmetic both forms are the same number; in FP32 the difference
 * of two rounded velocities loses the increment's bits once the parcel has nearly relaxed to
 * the carrier, the increment itself does not. */
template <class P, class V, int DEP>
__device__ __forceinline__ void evolve_parcel(const StepArgs<P, V>& a, P pos[3], V vel[3], V d,
                                              int32_t posI, V Ur[3], unsigned long long* acc,
                                              double* src, const Quant& qp, AmaxT<V>& amax,
                                              unsigned& ovf, bool& lost, int32_t& key,
                                              V dep[3])
{
    constexpr bool MIX = is_mixed<P, V>;
    const MeshK<P>& mesh = a.mesh;
    const PhysK<V>& ph = a.phys;
    const P dtP = a.dtP;
    /* mᵈ/ρᶜ = ρᵈ/ρᶜ·π·⌀³/6 (A:1280) */
    const V mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;
    /* drag factor 18 μ Δt/(ρᵈ ⌀²) (A:1294), times the drag multiplier */
    const V f = ((((V)18 * ph.mu) * a.dtV) / (ph.rho_d * (d * d))) * ph.alpha;
    P posNew[3] = {pos[0], pos[1], pos[2]};
    V velNew[3] = {vel[0], vel[1], vel[2]};
    V state0[3] = {vel[0], vel[1], vel[2]};                          /* A:1289 */
    V D[3] = {(V)0, (V)0, (V)0};                                     /* mixed: state0 - v */
    V Ulo[3];                                 /* mixed: Ur * fs_lo, formed once per cell */
#pragma unroll
    for (int k = 0; k < 3; ++k) Ulo[k] = MIX ? Ur[k] * a.fscale_lo : (V)0;
    bool bad = false;
    for (int t = 1; t <= ph.nsub; ++t) {                             /* A:1291 */
        V inc[3];
        if (ph.drag == 0) {
            if constexpr (MIX) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    inc[k] = (f * slip_lo<MIX>(Ur[k], a.fscale, Ulo[k], vel[k])) / ((V)1 + f);
                    velNew[k] = vel[k] + inc[k];
                }
            } else {
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    velNew[k] = (vel[k] + f * (Ur[k] * a.fscale)) / ((V)1 + f);  /* A:1295 */
            }
        } else {
            V du[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) du[k] = slip_lo<MIX>(Ur[k], a.fscale, Ulo[k], vel[k]);
            V mag = st_sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2]);
            V Re = (mag * d) * ph.rnu;
            V pw;
            if (sizeof(V) == 4) pw = (V)pow0687f_tab((float)Re);
            else pw = (V)st_pow0687((double)Re);
            V g = f * ((V)1 + (V)0.15 * pw);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                inc[k] = g * du[k];
                velNew[k] = vel[k] + inc[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) posNew[k] = pos[k] + (P)velNew[k] * dtP;  /* A:1296 */

        bool bnc[3] = {false, false, false};
        LocK ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);          /* A:1303 */
        if (bad) { lost = true; return; }
        if (ln.posI != posI || ln.part != 1) {                                   /* A:1306 */
            bnc[0] = (ln.I < 0) || (ln.I >= mesh.N[0]);
            bnc[1] = (ln.J < 0) || (ln.J >= mesh.N[1]);
            bnc[2] = (ln.K < 0) || (ln.K >= mesh.N[2]);
            /* hold position, mirror the old velocity, state0 -= 2 vel (A:1313-1329) */
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (bnc[k]) {
                    posNew[k] = pos[k];
                    velNew[k] = -vel[k];
                    if constexpr (!MIX) state0[k] -= (V)2 * vel[k];
                }
            }
            if (bnc[0] || bnc[1] || bnc[2]) {                                    /* A:1333-1335 */
                ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);
                if (bad) { lost = true; return; }
            }
        }
        if constexpr (MIX) {
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (!bnc[k]) D[k] -= inc[k];
        }
        if (t != ph.nsub && ln.posI != posI) {                                   /* A:1342-1348 */
            if (ln.part != 1 || ln.posI < 1 || ln.posI > mesh.nCells) { lost = true; return; }
            V di[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) di[k] = MIX ? mB * D[k] : mB * (state0[k] - velNew[k]);
            if (DEP == DEP_PROBE) {
#pragma unroll
                for (int k = 0; k < 3; ++k) track_max(di[k], amax);
            } else {
                deposit_direct<DEP, V>(di, (int64_t)(posI - 1), acc, src, qp, amax, ovf);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                state0[k] = velNew[k];
                D[k] = (V)0;
            }
            const V* Un = a.U + 3 * (int64_t)(ln.posI - 1);
            Ur[0] = __ldg(Un);
            Ur[1] = __ldg(Un + 1);
            Ur[2] = __ldg(Un + 2);
#pragma unroll
            for (int k = 0; k < 3; ++k) Ulo[k] = MIX ? Ur[k] * a.fscale_lo : (V)0;
            posI = ln.posI;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) { vel[k] = velNew[k]; pos[k] = posNew[k]; }
    }
    key = posI - 1;                                                              /* A:1361 */
#pragma unroll
    for (int k = 0; k < 3; ++k) dep[k] = MIX ? mB * D[k] : mB * (state0[k] - velNew[k]);
}

/* One substep (the benchmark configurations): evolve_particle! (A:1271-1365) with
 * nSteps = 1, where no intermediate deposit can happen and the final deposit goes to the
 * start cell.  A new position inside the mesh cannot meet a wall, so the reference's
 * relocation test (A:1303-1335) is only evaluated in full when the position left the index
 * range of some axis.  The deposit forms are those of evolve_parcel. */
template <class P, class V>
__device__ __forceinline__ void evolve_one(const StepArgs<P, V>& a, P pos[3], V vel[3], V d,
                                           int32_t posI, const V Ur[3], bool& lost, V dep[3])
{
    constexpr bool MIX = is_mixed<P, V>;
    const MeshK<P>& mesh = a.mesh;
    const PhysK<V>& ph = a.phys;
    const V mB = ((ph.rr * (V)3.14159265358979323846) * ((d * d) * d)) / (V)6;  /* A:1280 */
    const V f = ((((V)18 * ph.mu) * a.dtV) / (ph.rho_d * (d * d))) * ph.alpha; /* A:1294 */
    V velNew[3], inc[3];
    if (ph.drag == 0) {
        if constexpr (MIX) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                inc[k] = (f * slip<MIX>(Ur[k], a.fscale, a.fscale_lo, vel[k])) / ((V)1 + f);
                velNew[k] = vel[k] + inc[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; ++k)
                velNew[k] = (vel[k] + f * (Ur[k] * a.fscale)) / ((V)1 + f);     /* A:1295 */
        }
    } else {
        V du[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) du[k] = slip<MIX>(Ur[k], a.fscale, a.fscale_lo, vel[k]);
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
    P posNew[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) posNew[k] = pos[k] + (P)velNew[k] * a.dtP;              /* A:1296 */
    V state0[3] = {vel[0], vel[1], vel[2]};
    V D[3];
    if constexpr (MIX) {
#pragma unroll
        for (int k = 0; k < 3; ++k) D[k] = -inc[k];
    }
    /* floor(t) lies in [0, N) exactly when t does, so the fractional cell coordinates decide
     * whether the new position is inside without converting them */
    const P tx = (posNew[0] - mesh.origin[0]) * mesh.rD[0];
    const P ty = (posNew[1] - mesh.origin[1]) * mesh.rD[1];
    const P tz = (posNew[2] - mesh.origin[2]) * mesh.rD[2];
    if (!(tx >= (P)0 && tx < (P)mesh.N[0] && ty >= (P)0 && ty < (P)mesh.N[1] && tz >= (P)0 &&
          tz < (P)mesh.N[2])) {
        bool bad = false;
        LocK ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);                  /* A:1303 */
        if (bad) { lost = true; return; }
        if (ln.posI != posI || ln.part != 1) {                                          /* A:1306 */
            const bool bnc[3] = {(ln.I < 0) || (ln.I >= mesh.N[0]),
                                 (ln.J < 0) || (ln.J >= mesh.N[1]),
                                 (ln.K < 0) || (ln.K >= mesh.N[2])};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (bnc[k]) {
                    posNew[k] = pos[k];
                    velNew[k] = -vel[k];
                    if constexpr (MIX) D[k] = (V)0;
                    else state0[k] -= (V)2 * vel[k];
                }
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        pos[k] = posNew[k];
        vel[k] = velNew[k];
        if constexpr (MIX) dep[k] = mB * D[k];                                           /* A:1361 */
        else dep[k] = mB * (state0[k] - velNew[k]);
    }
}

}  // namespace st

#endif
