/*
 * adjoint_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU reference for the adjoint of the parcel step (no counterpart in the reference, which
 * has no adjoint): the gradient of an objective of the time-averaged momentum source,
 *   Sbar = (1/T) sum_n S_n,   S_n[c] = sum over parcels with cell c at step n of D_n,
 * with respect to the drag multiplier alpha, the diameter scale s and every parcel's initial
 * velocity, for Schiller-Naumann drag with one substep.  Cell ownership and wall-bounce
 * decisions are held fixed at those of the forward pass (frozen ownership): positions then
 * affect nothing downstream, and the adjoint state of a parcel is its velocity cotangent.
 *
 * Forward step n of one parcel (as evolve_parcel with nSteps = 1, A:1271-1365):
 *   u = U[c_n] fs_n,  d_e = s d,  f = 18 mu dt alpha / (rho_d d_e^2),
 *   du = u - v,  Re = |du| d_e rnu,  P = Re^0.687,  g = f (1 + 0.15 P)
 *   v'_k = v_k + g du_k         (k not bounced)        v'_k = -v_k   (k bounced)
 *   D_k  = m (v_k - v'_k)       (k not bounced)        D_k  = 0      (k bounced)
 * Reverse step, given a = dJ/dv' and G = dJ/dS_n[c_n] (the same for every n):
 *   w_k = a_k - m G_k (k not bounced),  Sw = sum_{k not bounced} w_k du_k,
 *   gamma = 0.10305 f P / |du|^2   (0 when du = 0),
 *   dJ/dv_j = [j not bounced]((1 - g) w_j + m G_j) - [j bounced] a_j - gamma du_j Sw
 *   dJ/dalpha += Sw g / alpha
 *   dJ/ds     += Sw (-2 g + 0.10305 f P) / s + (3/s) sum_k G_k D_k
 */
#ifndef ST_ADJOINT_ORACLE_HPP
#define ST_ADJOINT_ORACLE_HPP

#include <cmath>
#include <cstdint>
#include <vector>

#include "step_oracle.hpp"

namespace st_oracle {

/* What the forward pass fixes for the reverse pass: start cell (0-based) and bounce flags. */
struct Frozen {
    int32_t cell;
    uint8_t bounce;   /* bit k: component k bounced */
};

template <class V>
struct StepLocal {
    V mB, f, g, pw, mag2;
    V du[3];
    V velNew[3];
    V dep[3];
};

/* One forward step of one parcel.  With `replay` the cell and bounce decisions are taken
 * from `fz` instead of being computed (frozen ownership for finite differences); otherwise
 * they are computed as in evolve_parcel and written to `fz`. */
template <class P, class V>
bool adj_forward_step(const Params<P, V>& pr, P dtP, V dtV, const double* U, V fs, V fs_lo,
                      P pos[3], V vel[3], V dIn, Frozen& fz, bool replay, StepLocal<V>& o)
{
    constexpr bool MIX = mixed_mode<P, V>();
    const Mesh<P>& mesh = pr.mesh;
    const V d = dIn * pr.dscale;
    o.mB = ((pr.rhod_by_rhoc * (V)M_PI) * ((d * d) * d)) / (V)6;
    int32_t posI;
    if (replay) {
        posI = fz.cell + 1;
    } else {
        bool bad = false;
        Loc l0 = locate(mesh, pos[0], pos[1], pos[2], bad);
        if (bad || l0.partitionI != 1) return false;
        posI = l0.posI;
    }
    o.f = ((((V)18 * pr.mu) * dtV) / (pr.rho_d * (d * d))) * pr.alpha;
    for (int c = 0; c < 3; ++c)
        o.du[c] = slip_of<P, V>((V)U[3 * (int64_t)(posI - 1) + c], fs, fs_lo, vel[c]);
    o.mag2 = (o.du[0] * o.du[0] + o.du[1] * o.du[1]) + o.du[2] * o.du[2];
    V mag = std::sqrt(o.mag2);
    V Re = (mag * d) * pr.rnu;
    o.pw = (sizeof(V) == 4) ? (V)st_pow0687f((float)Re) : (V)st_pow0687((double)Re);
    o.g = o.f * ((V)1 + (V)0.15 * o.pw);
    P posNew[3];
    V inc[3];
    for (int c = 0; c < 3; ++c) {
        inc[c] = o.g * o.du[c];
        o.velNew[c] = vel[c] + inc[c];
        posNew[c] = pos[c] + (P)o.velNew[c] * dtP;
    }
    V state0[3] = {vel[0], vel[1], vel[2]};
    uint8_t b = 0;
    if (replay) {
        b = fz.bounce;
    } else {
        bool bad = false;
        Loc ln = locate(mesh, posNew[0], posNew[1], posNew[2], bad);
        if (bad) return false;
        if (ln.posI != posI || ln.partitionI != 1) {
            if (ln.I < 0 || ln.I >= mesh.N[0]) b |= 1;
            if (ln.J < 0 || ln.J >= mesh.N[1]) b |= 2;
            if (ln.K < 0 || ln.K >= mesh.N[2]) b |= 4;
        }
        fz.cell = posI - 1;
        fz.bounce = b;
    }
    for (int c = 0; c < 3; ++c) {
        if (b & (1 << c)) {
            posNew[c] = pos[c];
            o.velNew[c] = -vel[c];
            state0[c] -= (V)2 * vel[c];
        }
    }
    /* mixed precision deposits -m/rho_c times the increment, zero on a bounced component
     * (the deposit forms of evolve_parcel) */
    for (int c = 0; c < 3; ++c) {
        if (MIX) o.dep[c] = o.mB * ((b & (1 << c)) ? (V)0 : -inc[c]);
        else o.dep[c] = o.mB * (state0[c] - o.velNew[c]);
        pos[c] = posNew[c];
        vel[c] = o.velNew[c];
    }
    return true;
}

/* Reverse of one step.  `vel` is the velocity at the start of the step, `a` the cotangent
 * of the velocity after the step (in) and before it (out). */
template <class P, class V>
void adj_reverse_step(const Params<P, V>& pr, P dtP, V dtV, const double* U, V fs, V fs_lo,
                      V vel[3], V dIn, const Frozen& fz, const V G[3], V a[3], double& dalpha,
                      double& dscale)
{
    P pos[3] = {(P)0, (P)0, (P)0};
    V v[3] = {vel[0], vel[1], vel[2]};
    Frozen f2 = fz;
    StepLocal<V> o;
    adj_forward_step<P, V>(pr, dtP, dtV, U, fs, fs_lo, pos, v, dIn, f2, true, o);
    const uint8_t b = fz.bounce;
    V w[3];
    V Sw = (V)0;
    for (int k = 0; k < 3; ++k) {
        w[k] = (b & (1 << k)) ? (V)0 : a[k] - o.mB * G[k];
    }
    Sw = (w[0] * o.du[0] + w[1] * o.du[1]) + w[2] * o.du[2];
    const V gamma = o.mag2 > (V)0 ? (((V)0.10305 * o.f) * o.pw) / o.mag2 : (V)0;
    V an[3];
    for (int j = 0; j < 3; ++j) {
        V t = (b & (1 << j)) ? -a[j] : ((V)1 - o.g) * w[j] + o.mB * G[j];
        an[j] = t - (gamma * o.du[j]) * Sw;
    }
    for (int j = 0; j < 3; ++j) a[j] = an[j];
    dalpha += (double)(Sw * (o.g / pr.alpha));
    const V GD = (G[0] * o.dep[0] + G[1] * o.dep[1]) + G[2] * o.dep[2];
    dscale += (double)((Sw * ((V)-2 * o.g + ((V)0.10305 * o.f) * o.pw)) / pr.dscale +
                       ((V)3 / pr.dscale) * GD);
}

}  // namespace st_oracle

#endif
