/*
 * tet_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the face-walk relocation on unstructured tetrahedral meshes (no
 * counterpart in the reference, whose mesh is a uniform cuboid located by floor, A:663-697).
 * Used as the checker of the library's tet kernels (96^3 x 6 jittered tet workload included).
 *
 * Canonical order: every tet's vertex ids are first sorted in increasing order, its
 * neighbour list permuted with them (canonical_tets), so the three vertices of a face shared
 * by two tets appear in the same order in both.
 * Face planes (FP64): face f of tet (v0, v1, v2, v3) is opposite v_f, with vertices
 * (p, q, r) the other three in increasing order; n = (q - p) x (r - p), negated when
 * n . (v_f - p) > 0 so that it points out of the tet, and c = n . p; the signed distance of
 * a point x is s_f = n . x - c (sums left to right).  x is inside the closed tet when every
 * s_f <= 0.  Both tets of a shared face compute the same (n, c) bit for bit up to the exact
 * negation, so their signed distances are exact negatives of each other: a point is never
 * outside both of them (no walk can bounce between two tets).
 * Walk: from the current tet, if some s_f > 0 move across the face with the largest s_f
 * (first index on ties) to the neighbour; stop when inside, when the face is on the boundary
 * (neighbour -1: exit) or after the hop limit.
 * Step (project-defined; mirrors A:1271-1365 with the walk in place of locate): drag and
 * integration as on hex meshes; a new position outside the box [origin, ending] on axis k
 * keeps its old coordinate k and mirrors the old velocity component (A:1313-1329); the
 * walk then finds the new tet; deposits go to the tet of the last cell-velocity sample.
 */
#ifndef ST_TET_ORACLE_HPP
#define ST_TET_ORACLE_HPP

#include <cmath>
#include <cstdint>

#include "step_oracle.hpp"

namespace st_oracle {

struct TetMesh {
    int64_t nv, nt;
    const double* verts;    /* [nv][3] */
    const int32_t* tets;    /* [nt][4] */
    const int32_t* nbr;     /* [nt][4] */
    double origin[3], ending[3];
};

enum { WALK_OK = 0, WALK_EXIT = 1, WALK_HOPS = 2 };

/* Sorts each tet's vertex ids increasingly and permutes its neighbours with them. */
inline void canonical_tets(int64_t nt, const int32_t* tets, const int32_t* nbr, int32_t* tets_out,
                           int32_t* nbr_out)
{
    for (int64_t t = 0; t < nt; ++t) {
        int idx[4] = {0, 1, 2, 3};
        for (int i = 1; i < 4; ++i)
            for (int j = i; j > 0 && tets[4 * t + idx[j]] < tets[4 * t + idx[j - 1]]; --j) {
                const int tmp = idx[j];
                idx[j] = idx[j - 1];
                idx[j - 1] = tmp;
            }
        for (int k = 0; k < 4; ++k) {
            tets_out[4 * t + k] = tets[4 * t + idx[k]];
            nbr_out[4 * t + k] = nbr[4 * t + idx[k]];
        }
    }
}

/* Plane (n0, n1, n2, c) of face f of tet t. */
inline void tet_plane(const TetMesh& m, int32_t t, int f, double pl[4])
{
    static const int F[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    const double* v[4];
    for (int k = 0; k < 4; ++k) v[k] = m.verts + 3 * (int64_t)m.tets[4 * (int64_t)t + k];
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
    pl[0] = n0;
    pl[1] = n1;
    pl[2] = n2;
    pl[3] = (n0 * p[0] + n1 * p[1]) + n2 * p[2];
}

inline void tet_signed(const TetMesh& m, int32_t t, const double x[3], double s[4])
{
    for (int f = 0; f < 4; ++f) {
        double pl[4];
        tet_plane(m, t, f, pl);
        s[f] = ((pl[0] * x[0] + pl[1] * x[1]) + pl[2] * x[2]) - pl[3];
    }
}

inline int32_t tet_walk(const TetMesh& m, int32_t t, const double x[3], int hop_limit,
                        int& status, int& hops)
{
    hops = 0;
    for (;;) {
        double s[4];
        tet_signed(m, t, x, s);
        int fb = 0;
        for (int f = 1; f < 4; ++f)
            if (s[f] > s[fb]) fb = f;
        if (!(s[fb] > 0.0)) { status = WALK_OK; return t; }
        const int32_t nb = m.nbr[4 * (int64_t)t + fb];
        if (nb < 0) { status = WALK_EXIT; return t; }
        if (hops >= hop_limit) { status = WALK_HOPS; return t; }
        t = nb;
        ++hops;
    }
}

/* One call of the step for one parcel on a tet mesh (positions in double).  Returns false
 * if the parcel was lost (walk exit or hop limit); the state is then unchanged.  The velocity
 * update and deposit forms are those of evolve_parcel in step_oracle.hpp (mixed precision:
 * compensated slip and the carried D = state0 - v). */
template <class V>
bool evolve_parcel_tet(const TetMesh& m, const Params<double, V>& pr, double dtP, V dtV,
                       const double* U, V fscale, V fscale_lo, double pos0[3], V vel0[3],
                       int32_t& cell, V dIn, int hop_limit, Sink<V>& sink, int64_t* hop_hist)
{
    constexpr bool MIX = mixed_mode<double, V>();
    const V d = dIn * pr.dscale;
    const V mByRho = ((pr.rhod_by_rhoc * (V)M_PI) * ((d * d) * d)) / (V)6;
    double pos[3] = {pos0[0], pos0[1], pos0[2]};
    V vel[3] = {vel0[0], vel0[1], vel0[2]};
    double posNew[3] = {pos[0], pos[1], pos[2]};
    V velNew[3] = {vel[0], vel[1], vel[2]};
    int32_t cur = cell;
    V Ur[3];
    for (int c = 0; c < 3; ++c) Ur[c] = (V)U[3 * (int64_t)cur + c];
    V state0[3] = {vel[0], vel[1], vel[2]};
    V D[3] = {0, 0, 0};
    const V f = ((((V)18 * pr.mu) * dtV) / (pr.rho_d * (d * d))) * pr.alpha;
    int32_t tNew = cur;
    for (int t = 1; t <= pr.nsub; ++t) {
        V inc[3] = {0, 0, 0};
        if (pr.drag == DRAG_STOKES_IMPLICIT) {
            if (MIX) {
                for (int c = 0; c < 3; ++c) {
                    inc[c] = (f * slip_of<double, V>(Ur[c], fscale, fscale_lo, vel[c])) / ((V)1 + f);
                    velNew[c] = vel[c] + inc[c];
                }
            } else {
                for (int c = 0; c < 3; ++c)
                    velNew[c] = (vel[c] + f * (Ur[c] * fscale)) / ((V)1 + f);
            }
        } else {
            V du[3];
            for (int c = 0; c < 3; ++c) du[c] = slip_of<double, V>(Ur[c], fscale, fscale_lo, vel[c]);
            V mag = std::sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2]);
            V Re = (mag * d) * pr.rnu;
            V pw = (sizeof(V) == 4) ? (V)st_pow0687f((float)Re) : (V)st_pow0687((double)Re);
            V g = f * ((V)1 + (V)0.15 * pw);
            for (int c = 0; c < 3; ++c) {
                inc[c] = g * du[c];
                velNew[c] = vel[c] + inc[c];
            }
        }
        for (int c = 0; c < 3; ++c) posNew[c] = pos[c] + (double)velNew[c] * dtP;
        for (int c = 0; c < 3; ++c) {
            if (posNew[c] < m.origin[c] || posNew[c] > m.ending[c]) {
                posNew[c] = pos[c];
                velNew[c] = -vel[c];
                if (!MIX) state0[c] -= (V)2 * vel[c];
            } else if (MIX) {
                D[c] -= inc[c];
            }
        }
        int status = WALK_OK, hops = 0;
        tNew = tet_walk(m, tNew, posNew, hop_limit, status, hops);
        if (status != WALK_OK) return false;
        if (hop_hist) ++hop_hist[hops < 7 ? hops : 7];
        if (t != pr.nsub && tNew != cur) {
            if (MIX)
                sink.deposit(cur + 1, mByRho * D[0], mByRho * D[1], mByRho * D[2]);
            else
                sink.deposit(cur + 1, mByRho * (state0[0] - velNew[0]),
                             mByRho * (state0[1] - velNew[1]), mByRho * (state0[2] - velNew[2]));
            for (int c = 0; c < 3; ++c) {
                state0[c] = velNew[c];
                D[c] = 0;
            }
            for (int c = 0; c < 3; ++c) Ur[c] = (V)U[3 * (int64_t)tNew + c];
            cur = tNew;
        }
        for (int c = 0; c < 3; ++c) { vel[c] = velNew[c]; pos[c] = posNew[c]; }
    }
    if (MIX)
        sink.deposit(cur + 1, mByRho * D[0], mByRho * D[1], mByRho * D[2]);
    else
        sink.deposit(cur + 1, mByRho * (state0[0] - velNew[0]), mByRho * (state0[1] - velNew[1]),
                     mByRho * (state0[2] - velNew[2]));
    for (int c = 0; c < 3; ++c) { pos0[c] = posNew[c]; vel0[c] = velNew[c]; }
    cell = tNew;
    return true;
}

}  // namespace st_oracle

#endif
