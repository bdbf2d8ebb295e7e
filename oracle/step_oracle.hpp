/*
 * step_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of SCALE-TRACK's Lagrangian parcel step, used by the tests, by
 * __graft_entry__.smoke() and by the CPU baseline leg of bench.py as the checker.  It is
 * never part of the shipped library and the library never calls it.
 *
 * Parity status: the reference (Julia + CUDA.jl, embedded in an OpenFOAM solver) cannot run
 * in this environment (no Julia, no OpenFOAM, no MPI) and it ships no tests, golden vectors
 * or fixtures.  This restatement is therefore pinned by analytic known-answer tests (Stokes
 * relaxation, wall-bounce symmetry, momentum bookkeeping) and by a second, independent
 * line-by-line restatement in Python (tests/golden/gen_golden.py: numpy float32 scalars and
 * Python binary64 floats, for the FP32, mixed and FP64 modes) whose outputs are committed as
 * fixtures.  In the strict sense the parity is "unpinned" against the running
 * reference.
 *
 * Reference file cited as A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
 *
 * Template parameters: P is the position type, V the velocity/drag type.
 *   P = V = float   : the reference's own arithmetic (const scalar = Float32, A:172)
 *   P = double, V = float  : mixed precision (FP64 positions, FP32 drag and velocity)
 *   P = V = double  : all-FP64 oracle
 * Build with -ffp-contract=off: Julia does not contract a*b+c into fma, and neither do we.
 */
#ifndef ST_STEP_ORACLE_HPP
#define ST_STEP_ORACLE_HPP

#include <cmath>
#include <cstdint>
#include <climits>

#include "../scale-track_b200/csrc/st_pow.h"

namespace st_oracle {

enum { DRAG_STOKES_IMPLICIT = 0, DRAG_SN_EXPLICIT = 1 };

/* Uniform cuboid mesh with decomposition (1,1,1): A:222-270.
 * construct_mesh computes L = ending - origin, Delta = L ./ N and rDelta = 1 ./ Delta in
 * Float64 and stores them as Float32 (A:237-240, Mesh fields are ScalarVec). */
template <class P>
struct Mesh {
    int32_t N[3];
    P origin[3];
    P rDelta[3];
    int32_t NxNy;   /* partitionNxTimesNy with one partition (A:253) */
    int64_t nCells;
};

template <class P>
Mesh<P> make_mesh(const int32_t n[3], const double origin[3], const double ending[3])
{
    Mesh<P> m;
    for (int a = 0; a < 3; ++a) {
        m.N[a] = n[a];
        m.origin[a] = (P)origin[a];
        double L = ending[a] - origin[a];
        double D = L / (double)n[a];
        m.rDelta[a] = (P)(1.0 / D);
    }
    m.NxNy = n[0] * n[1];
    m.nCells = (int64_t)n[0] * n[1] * n[2];
    return m;
}

/* floor(label, v) (A:668-670): Julia throws InexactError outside Int32; we report it. */
template <class T>
inline int32_t floor_label(T v, bool& bad)
{
    T f = std::floor(v);
    if (!(f >= (T)-2147483648.0 && f < (T)2147483648.0)) {
        bad = true;
        return 0;
    }
    return (int32_t)f;
}

struct Loc {
    int32_t I, J, K;
    int32_t posI;        /* 1-based linear cell index as in the reference */
    int32_t partitionI;  /* 1-based partition index */
};

/* locate_ijk + locate (A:663-697) with decomposition = (1,1,1), partitionN = N:
 *   iGlobal = floor((x - origin) * rDelta); (iPartition, iLocal) = divrem(iGlobal, N)
 *   partitionI = |kP|*1 + |jP|*1 + |iP| + 1 ; posI = |kL|*NxNy + |jL|*Nx + |iL| + 1
 * divrem truncates toward zero, like C++ '/' and '%'. */
template <class P>
inline Loc locate(const Mesh<P>& m, P x, P y, P z, bool& bad)
{
    Loc r;
    r.I = floor_label((x - m.origin[0]) * m.rDelta[0], bad);
    r.J = floor_label((y - m.origin[1]) * m.rDelta[1], bad);
    r.K = floor_label((z - m.origin[2]) * m.rDelta[2], bad);
    int32_t iP = r.I / m.N[0], iL = r.I % m.N[0];
    int32_t jP = r.J / m.N[1], jL = r.J % m.N[1];
    int32_t kP = r.K / m.N[2], kL = r.K % m.N[2];
    r.partitionI = std::abs(kP) * 1 + std::abs(jP) * 1 + std::abs(iP) + 1;
    r.posI = std::abs(kL) * m.NxNy + std::abs(jL) * m.N[0] + std::abs(iL) + 1;
    return r;
}

/* Physical constants in the parcel's arithmetic type.  Chunk stores mu_c, rho_d and
 * rho_d/rho_c as Float32 (A:330-345, A:1608: ρᵈ/ρᶜ is formed in Float64 then converted). */
template <class P, class V>
struct Params {
    Mesh<P> mesh;
    V mu;           /* carrier dynamic viscosity */
    V rho_d;        /* parcel density */
    V rhod_by_rhoc; /* rho_d / rho_c */
    V nu;           /* carrier kinematic viscosity mu/rho_c */
    V rnu;          /* rho_c/mu_c: Schiller-Naumann Re = |u - v| d rnu */
    V alpha;        /* drag multiplier (1 reproduces the reference) */
    V dscale;       /* diameter scale (1 reproduces the reference) */
    int drag;
    int nsub;
};

template <class P, class V>
Params<P, V> make_params(const int32_t n[3], const double origin[3], const double ending[3],
                         double mu_c, double rho_c, double rho_d, int drag, int nsub,
                         double alpha, double dscale)
{
    Params<P, V> p;
    p.mesh = make_mesh<P>(n, origin, ending);
    p.mu = (V)mu_c;
    p.rho_d = (V)rho_d;
    p.rhod_by_rhoc = (V)(rho_d / rho_c);
    p.nu = (V)(mu_c / rho_c);
    p.rnu = (V)(rho_c / mu_c);
    p.alpha = (V)alpha;
    p.dscale = (V)dscale;
    p.drag = drag;
    p.nsub = nsub;
    return p;
}

/* Deposit sink interface: called with the 1-based cell and the three components of
 * m/rho_c * (state0 - velocity) (A:703-708 with '+=' semantics, A:714-725 on the GPU). */
template <class V>
struct Sink {
    virtual void deposit(int32_t posI, V d0, V d1, V d2) = 0;
    virtual ~Sink() {}
};

/* Mixed precision (P = double, V = float) is project-defined: the reference computes in
 * Float32 only.  Two of its operations are arranged so that the result stays close to the
 * all-FP64 step when a parcel has nearly relaxed to the carrier:
 *   slip   u_c - v = fma(U, fs_hi, -v) + U * fs_lo, with fs = fs_hi + fs_lo the fluid
 *          factor split into a float and its FP64 remainder (the product U*fs_hi is exact
 *          inside the fma);
 *   source D = state0 - v is carried instead of state0: every substep subtracts its velocity
 *          increment, a component that bounces keeps its D, and a deposit is m/rho_c * D.
 * P = V (FP32 reference mode and all-FP64) follow the reference's form exactly. */
template <class P, class V>
constexpr bool mixed_mode() { return sizeof(P) == 8 && sizeof(V) == 4; }

template <class P, class V>
inline V slip_of(V U, V fs, V fs_lo, V v)
{
    if (mixed_mode<P, V>()) return std::fma(U, fs, -v) + U * fs_lo;
    return U * fs - v;
}

/* The fluid factor of step s (1 when there is none) as a V value and, in mixed precision,
 * its FP64 remainder. */
template <class P, class V>
inline void split_factor(const double* fscale, int s, V& hi, V& lo)
{
    const double f = fscale ? fscale[s] : 1.0;
    hi = (V)f;
    lo = mixed_mode<P, V>() ? (V)(f - (double)hi) : (V)0;
}

/* evolve_particle! (A:1271-1365) for one parcel over one call of the step.
 * Returns false if the parcel could not be located (the reference would index out of
 * bounds or throw); the state is then left unchanged and nothing is deposited.
 * fscale_lo is the FP64 remainder of the fluid factor (mixed precision; 0 otherwise). */
template <class P, class V>
bool evolve_parcel(const Params<P, V>& pr, P dtP, V dtV, const double* U, V fscale,
                   V fscale_lo, P& X, P& Y, P& Z, V& Uv, V& Vv, V& Wv, V dIn, Sink<V>& sink)
{
    constexpr bool MIX = mixed_mode<P, V>();
    const Mesh<P>& mesh = pr.mesh;
    const V d = dIn * pr.dscale;
    /* mᵈByρᶜ = ρᵈByρᶜ*π*⌀^3/6 (A:1280): left fold, ⌀^3 = ⌀*⌀*⌀ (literal_pow), π rounded to V */
    const V mByRho = ((pr.rhod_by_rhoc * (V)M_PI) * ((d * d) * d)) / (V)6;
    P pos[3] = {X, Y, Z};
    V vel[3] = {Uv, Vv, Wv};
    P posNew[3] = {X, Y, Z};
    V velNew[3] = {Uv, Vv, Wv};

    bool bad = false;
    Loc L0 = locate(mesh, pos[0], pos[1], pos[2], bad);            /* A:1286 */
    if (bad || L0.partitionI != 1 || L0.posI < 1 || L0.posI > mesh.nCells) return false;
    int32_t posI = L0.posI;
    int32_t partitionI = L0.partitionI;
    V Ur[3];                                                          /* A:1288 (raw U) */
    for (int c = 0; c < 3; ++c) Ur[c] = (V)U[3 * (int64_t)(posI - 1) + c];
    V state0[3] = {vel[0], vel[1], vel[2]};                          /* A:1289 */
    V D[3] = {0, 0, 0};                                              /* mixed: state0 - vel */

    /* dragFactor = 18*μᶜ*Δt/(ρᵈ*⌀^2) (A:1294) */
    const V f = ((((V)18 * pr.mu) * dtV) / (pr.rho_d * (d * d))) * pr.alpha;

    for (int t = 1; t <= pr.nsub; ++t) {                            /* A:1291 */
        V inc[3] = {0, 0, 0};
        if (pr.drag == DRAG_STOKES_IMPLICIT) {
            if (MIX) {
                /* the same update as an increment: v' = v + f (u - v)/(1 + f) */
                for (int c = 0; c < 3; ++c) {
                    inc[c] = (f * slip_of<P, V>(Ur[c], fscale, fscale_lo, vel[c])) / ((V)1 + f);
                    velNew[c] = vel[c] + inc[c];
                }
            } else {
                /* velNew = (vel + f*uᶜ)/(1 + f), uᶜ = U*fscale (A:1288, A:1295) */
                for (int c = 0; c < 3; ++c)
                    velNew[c] = (vel[c] + f * (Ur[c] * fscale)) / ((V)1 + f);
            }
        } else {
            /* Schiller-Naumann, explicit Euler (project-defined; no reference code):
             * v' = v + f (1 + 0.15 Re^0.687) (u - v), Re = |u - v| d (1/nu) */
            V du[3];
            for (int c = 0; c < 3; ++c) du[c] = slip_of<P, V>(Ur[c], fscale, fscale_lo, vel[c]);
            V mag = std::sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2]);
            V Re = (mag * d) * pr.rnu;
            V pw = (sizeof(V) == 4) ? (V)st_pow0687f((float)Re) : (V)st_pow0687((double)Re);
            V g = f * ((V)1 + (V)0.15 * pw);
            for (int c = 0; c < 3; ++c) {
                inc[c] = g * du[c];
                velNew[c] = vel[c] + inc[c];
            }
        }
        /* posNew = pos + velNew*Δt (A:1296) */
        for (int c = 0; c < 3; ++c) posNew[c] = pos[c] + (P)velNew[c] * dtP;

        Loc Ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);  /* A:1303 */
        if (bad) return false;
        int32_t posNewI = Ln.posI;
        int32_t partitionNewI = Ln.partitionI;

        bool bnc[3] = {false, false, false};
        if (posNewI != posI || partitionNewI != partitionI) {          /* A:1306 */
            bnc[0] = (Ln.I < 0) || (Ln.I >= mesh.N[0]);               /* A:1309-1311 */
            bnc[1] = (Ln.J < 0) || (Ln.J >= mesh.N[1]);
            bnc[2] = (Ln.K < 0) || (Ln.K >= mesh.N[2]);
            /* hold the position component, mirror the OLD velocity, correct state0
             * by -2*vel (update_at_boundary!, A:731-736; A:1313-1329) */
            for (int c = 0; c < 3; ++c) {
                if (bnc[c]) {
                    posNew[c] = pos[c];
                    velNew[c] = -vel[c];
                    if (!MIX) state0[c] -= (V)2 * vel[c];
                }
            }
            if (bnc[0] || bnc[1] || bnc[2]) {                            /* A:1333-1335 */
                Ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);
                if (bad) return false;
                posNewI = Ln.posI;
                partitionNewI = Ln.partitionI;
            }
            /* A:1337-1340 re-points to eulerianArr[partitionI] (the old one): a no-op
             * with a single partition.  partitionI keeps its initial value: the reference
             * never reassigns it. */
        }
        if (MIX)
            for (int c = 0; c < 3; ++c)
                if (!bnc[c]) D[c] -= inc[c];
        if (t != pr.nsub && posNewI != posI) {                           /* A:1342-1348 */
            if (partitionNewI != 1 || posNewI < 1 || posNewI > mesh.nCells) return false;
            if (MIX)
                sink.deposit(posI, mByRho * D[0], mByRho * D[1], mByRho * D[2]);
            else
                sink.deposit(posI, mByRho * (state0[0] - velNew[0]),
                             mByRho * (state0[1] - velNew[1]),
                             mByRho * (state0[2] - velNew[2]));
            for (int c = 0; c < 3; ++c) {
                state0[c] = velNew[c];
                D[c] = 0;
            }
            for (int c = 0; c < 3; ++c) Ur[c] = (V)U[3 * (int64_t)(posNewI - 1) + c];
            posI = posNewI;
        }
        for (int c = 0; c < 3; ++c) { vel[c] = velNew[c]; pos[c] = posNew[c]; }
    }

    X = posNew[0]; Y = posNew[1]; Z = posNew[2];                        /* A:1355-1360 */
    Uv = velNew[0]; Vv = velNew[1]; Wv = velNew[2];
    if (MIX)                                                            /* A:1361 */
        sink.deposit(posI, mByRho * D[0], mByRho * D[1], mByRho * D[2]);
    else
        sink.deposit(posI, mByRho * (state0[0] - velNew[0]),
                     mByRho * (state0[1] - velNew[1]),
                     mByRho * (state0[2] - velNew[2]));
    return true;
}

/* ---------------------------------------------------------------------------------------
 * Fixed-point model of the library's deterministic deposit.
 *
 * Each deposit component is scaled by 2^-L and rounded to the nearest integer (ties to
 * even); integer sums do not depend on the order of addition, so the library's result is
 * reproducible and this model reproduces it bit for bit.  L follows the largest deposit of
 * the previous step (or of a read-only probe pass for the first step):
 *   e      = smallest integer with |dep| < 2^e   (frexp exponent)
 *   L_next = emax - H,  H = 62 - G - nb  (one 64-bit limb)  or  62 - G  (two limbs)
 *   nb     = ceil(log2(number of deposits bound)), G = 8 bits of growth allowance.
 * A deposit with e - L > H + G would overflow and is reported instead of added.
 * ------------------------------------------------------------------------------------- */
static const int QUANT_GROWTH_BITS = 8;
static const int EXP_NONE = -100000;

inline int quant_nbits(int64_t n_deposit_bound)
{
    int nb = 1;
    while (nb < 62 && ((int64_t)1 << nb) < n_deposit_bound) ++nb;
    return nb;
}

inline int quant_headroom(int limbs, int64_t n_deposit_bound)
{
    return limbs == 1 ? 62 - QUANT_GROWTH_BITS - quant_nbits(n_deposit_bound)
                      : 62 - QUANT_GROWTH_BITS;
}

/* x * 2^k, exact unless the result leaves the normal range */
inline double ldexp2(double x, int k)
{
    int k1 = k / 2;
    int k2 = k - k1;
    return (x * st_pow2i(k1)) * st_pow2i(k2);
}

inline int exp_of(double a)  /* smallest e with |a| < 2^e, a != 0 */
{
    int e;
    (void)std::frexp(a, &e);
    return e;
}

}  // namespace st_oracle

#endif
