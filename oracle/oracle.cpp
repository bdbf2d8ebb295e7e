/*
 * oracle.cpp -- TEST INFRASTRUCTURE ONLY: C entry points around step_oracle.hpp so that the
 * Python tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg can run the CPU
 * restatement through ctypes.  Nothing in the shipped library links or calls this file.
 *
 * The driver loop follows the reference's CPU executor (A:818-823: a serial loop over the
 * parcels of a chunk calling evolve_particle!) with the time step handling of A:487-502 and
 * A:1260 (the substep is Δt/nSteps, with Δt held in the parcel precision).
 */
#include <cstdint>
#include <cstring>
#include <climits>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "step_oracle.hpp"
#include "adjoint_oracle.hpp"
#include "tet_oracle.hpp"
#include "../scale-track_b200/csrc/st_init.h"

using namespace st_oracle;

extern "C" {

typedef struct oracle_cfg {
    int32_t n[3];
    double origin[3];
    double ending[3];
    double mu_c;
    double rho_c;
    double rho_d;
    int32_t drag;         /* 0 Stokes implicit (reference), 1 Schiller-Naumann explicit */
    int32_t precision;    /* 0 FP32 (reference), 1 mixed, 2 FP64 */
    int32_t n_substeps;   /* 10 in the reference (A:1260) */
    int32_t quant_limbs;  /* 1 or 2: fixed-point model of the deterministic deposit */
    double drag_multiplier;
    double diameter_scale;
    int64_t deposit_bound;  /* parcels whose deposits share one fixed-point sum (all ranks of
                               a sharded run); 0: the parcels of this call */
} oracle_cfg;

}  // extern "C"

namespace {

struct Acc {
    double* seq = nullptr;       /* FP64 sum of the deposits, parcel order */
    int64_t* q1 = nullptr;       /* one-limb fixed point */
    int64_t* hi = nullptr;       /* two-limb fixed point: high part */
    uint64_t* lo = nullptr;      /* two-limb fixed point: low 32 bits */
    int limbs = 1;
    int L = 0;
    int H = 0;
    bool parallel = false;
};

template <class V>
struct AccSink : Sink<V> {
    Acc* a;
    bool quant;
    int emax = EXP_NONE;
    int64_t overflow = 0;
    int64_t count = 0;
    explicit AccSink(Acc* acc, bool q) : a(acc), quant(q) {}
    void deposit(int32_t posI, V d0, V d1, V d2) override
    {
        const int64_t base = 3 * (int64_t)(posI - 1);
        const V comp[3] = {d0, d1, d2};
        ++count;
        for (int k = 0; k < 3; ++k) {
            double dv = (double)comp[k];
            if (a->seq) {
                if (a->parallel) {
#pragma omp atomic
                    a->seq[base + k] += dv;
                } else {
                    a->seq[base + k] += dv;
                }
            }
            if (!quant || dv == 0.0) continue;
            if (!std::isfinite(dv)) { ++overflow; continue; }
            int e = exp_of(dv);
            emax = std::max(emax, e);
            if (e - a->L > a->H + QUANT_GROWTH_BITS) { ++overflow; continue; }
            int64_t q = std::llrint(ldexp2(dv, -a->L));
            if (!a->q1 && !a->hi) continue;          /* probe pass */
            if (a->limbs == 1) {
                uint64_t* p = reinterpret_cast<uint64_t*>(a->q1 + base + k);
                if (a->parallel) {
#pragma omp atomic
                    *p += (uint64_t)q;
                } else {
                    *p += (uint64_t)q;
                }
            } else {
                int64_t h = q >> 32;
                uint64_t l = (uint64_t)q & 0xffffffffULL;
                if (a->parallel) {
#pragma omp atomic
                    a->hi[base + k] += h;
#pragma omp atomic
                    a->lo[base + k] += l;
                } else {
                    a->hi[base + k] += h;
                    a->lo[base + k] += l;
                }
            }
        }
    }
};

template <class P, class V>
int run(const oracle_cfg* cfg, int64_t np, double* xyz, double* uvw, const double* d,
        const double* U, int nsteps, double dt, const double* fscale, double* src_seq,
        double* src_quant, int32_t* cells, int32_t* scale_io, int64_t* stats, int nthreads,
        int64_t* acc_out)
{
    Params<P, V> pr = make_params<P, V>(cfg->n, cfg->origin, cfg->ending, cfg->mu_c, cfg->rho_c,
                                        cfg->rho_d, cfg->drag, cfg->n_substeps,
                                        cfg->drag_multiplier, cfg->diameter_scale);
    const int64_t nC = pr.mesh.nCells;
    std::vector<P> X(np), Y(np), Z(np);
    std::vector<V> Uu(np), Vv(np), Ww(np), D(np);
    for (int64_t i = 0; i < np; ++i) {
        X[i] = (P)xyz[i]; Y[i] = (P)xyz[np + i]; Z[i] = (P)xyz[2 * np + i];
        Uu[i] = (V)uvw[i]; Vv[i] = (V)uvw[np + i]; Ww[i] = (V)uvw[2 * np + i];
        D[i] = (V)d[i];
    }
    /* Time step in the parcel precision: Time.Δt is a Float32 (A:324-327), the substep is
     * Δt/nSteps (A:1260).  Mixed precision keeps the substep in FP64 for positions. */
    const P dtP = (P)dt / (P)cfg->n_substeps;
    const V dtV = (V)dtP;

    const bool quant = (src_quant != nullptr);
    const int limbs = cfg->quant_limbs == 2 ? 2 : 1;
    std::vector<int64_t> q1, hi;
    std::vector<uint64_t> lo;
    std::vector<double> seq;
    if (quant) {
        if (limbs == 1) q1.assign(3 * nC, 0);
        else { hi.assign(3 * nC, 0); lo.assign(3 * nC, 0); }
    }
    seq.assign(src_seq ? 3 * nC : 0, 0.0);
    const int64_t nbound =
        std::max<int64_t>(2, std::max<int64_t>(np, cfg->deposit_bound) * (int64_t)cfg->n_substeps);
    const int H = quant_headroom(limbs, nbound);
    int L = scale_io ? *scale_io : INT_MIN;
    int emax_last = EXP_NONE;
    /* nsteps == 0 with scale INT_MIN: the probe of the next step only (its exponent in
     * stats[3]); the state is not advanced */
    const bool probe_only = (nsteps == 0 && quant && L == INT_MIN);
    int64_t lost = 0, overflow = 0;

#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    const bool par = nthreads != 1;

    for (int s = 0; s < (probe_only ? 1 : nsteps); ++s) {
        V fs, fs_lo;
        split_factor<P, V>(fscale, s, fs, fs_lo);
        if (quant && L == INT_MIN) {
            /* probe: the deposits of this step without committing the state */
            Acc pa;
            pa.limbs = limbs; pa.L = 0; pa.H = 1 << 20; pa.parallel = false;
            int emax = EXP_NONE;
#pragma omp parallel for schedule(static) reduction(max : emax) if (par)
            for (int64_t i = 0; i < np; ++i) {
                AccSink<V> sk(&pa, true);
                P x = X[i], y = Y[i], z = Z[i];
                V u = Uu[i], v = Vv[i], w = Ww[i];
                evolve_parcel<P, V>(pr, dtP, dtV, U, fs, fs_lo, x, y, z, u, v, w, D[i], sk);
                emax = std::max(emax, sk.emax);
            }
            L = (emax == EXP_NONE) ? -H : emax - H;
            if (probe_only) {
                emax_last = emax;
                break;
            }
        }
        const bool last = (s == nsteps - 1);
        Acc acc;
        acc.limbs = limbs; acc.L = L; acc.H = H; acc.parallel = par;
        if (src_seq) { std::fill(seq.begin(), seq.end(), 0.0); acc.seq = seq.data(); }
        if (quant) {
            if (limbs == 1) { std::fill(q1.begin(), q1.end(), 0); acc.q1 = q1.data(); }
            else {
                std::fill(hi.begin(), hi.end(), 0); std::fill(lo.begin(), lo.end(), 0);
                acc.hi = hi.data(); acc.lo = lo.data();
            }
        }
        int emax = EXP_NONE;
        int64_t lost_s = 0, ovf_s = 0;
#pragma omp parallel for schedule(static) reduction(max : emax) reduction(+ : lost_s, ovf_s) if (par)
        for (int64_t i = 0; i < np; ++i) {
            AccSink<V> sk(&acc, quant);
            if (!evolve_parcel<P, V>(pr, dtP, dtV, U, fs, fs_lo, X[i], Y[i], Z[i], Uu[i], Vv[i],
                                     Ww[i], D[i], sk))
                ++lost_s;
            emax = std::max(emax, sk.emax);
            ovf_s += sk.overflow;
        }
        lost += lost_s;
        overflow += ovf_s;
        if (last && quant) {
            for (int64_t j = 0; j < 3 * nC; ++j) {
                double v;
                if (limbs == 1) {
                    v = (double)q1[j];
                } else {
                    int64_t h = hi[j] + (int64_t)(lo[j] >> 32);
                    uint64_t l = lo[j] & 0xffffffffULL;
                    v = (double)h * 4294967296.0 + (double)l;
                }
                src_quant[j] = ldexp2(v, L);
            }
        }
        if (last && quant && acc_out) {
            for (int64_t j = 0; j < 3 * nC; ++j) {
                if (limbs == 1) {
                    acc_out[j] = q1[j];
                } else {  /* the library's two-limb layout: [hi, lo] per component */
                    acc_out[2 * j] = hi[j];
                    acc_out[2 * j + 1] = (int64_t)lo[j];
                }
            }
        }
        emax_last = emax;
        if (quant && emax != EXP_NONE) L = emax - H;
    }
    if (src_seq) std::memcpy(src_seq, seq.data(), sizeof(double) * 3 * nC);
    if (scale_io) *scale_io = L;

    for (int64_t i = 0; i < np; ++i) {
        xyz[i] = (double)X[i]; xyz[np + i] = (double)Y[i]; xyz[2 * np + i] = (double)Z[i];
        uvw[i] = (double)Uu[i]; uvw[np + i] = (double)Vv[i]; uvw[2 * np + i] = (double)Ww[i];
        if (cells) {
            bool bad = false;
            Loc l = locate(pr.mesh, X[i], Y[i], Z[i], bad);
            cells[i] = (bad || l.partitionI != 1) ? -1 : l.posI - 1;
        }
    }
    if (stats) { stats[0] = lost; stats[1] = overflow; stats[2] = H; stats[3] = emax_last; }
    return (int)(lost > 0 ? 1 : 0) | (overflow > 0 ? 2 : 0);
}

}  // namespace

extern "C" {

/* Runs nsteps steps of the parcel step on the CPU.
 *  xyz, uvw : [3][np] SoA, in/out (values are converted to the configured precision)
 *  d        : [np] diameters;  U: [nCells][3] cell velocity (AoS, the exchange layout)
 *  fscale   : per-step factor on U, or NULL for 1
 *  src_seq  : [nCells][3] FP64 sum of the last step's deposits in parcel order, or NULL
 *  src_quant: [nCells][3] fixed-point model of the library's deterministic deposit, or NULL
 *  cells    : [np] 0-based owning cell after the last step (-1 if lost), or NULL
 *  scale_io : in: scale exponent for the first step (INT_MIN: probe); out: for the next step
 *  stats    : [4] lost parcels, overflowing deposits, headroom bits H, largest-deposit
 *             exponent of the last step (or of the probe when nsteps == 0), or NULL
 *  acc_out  : raw fixed-point accumulators of the last step (int64 [nCells*3], two limbs:
 *             [nCells*3][hi, lo]), or NULL
 * nsteps == 0 with *scale_io == INT_MIN runs the probe of the first step only.
 * Returns 0, or a bit set: 1 = some parcel could not be located, 2 = deposit overflow. */
int oracle_run(const oracle_cfg* cfg, int64_t np, double* xyz, double* uvw, const double* d,
               const double* U, int nsteps, double dt, const double* fscale, double* src_seq,
               double* src_quant, int32_t* cells, int32_t* scale_io, int64_t* stats, int nthreads,
               int64_t* acc_out)
{
    switch (cfg->precision) {
    case 0:
        return run<float, float>(cfg, np, xyz, uvw, d, U, nsteps, dt, fscale, src_seq, src_quant,
                                 cells, scale_io, stats, nthreads, acc_out);
    case 1:
        return run<double, float>(cfg, np, xyz, uvw, d, U, nsteps, dt, fscale, src_seq, src_quant,
                                  cells, scale_io, stats, nthreads, acc_out);
    case 2:
        return run<double, double>(cfg, np, xyz, uvw, d, U, nsteps, dt, fscale, src_seq,
                                   src_quant, cells, scale_io, stats, nthreads, acc_out);
    default:
        return -1;
    }
}

/* 0-based owning cell of each position (locate, A:680-693), -1 if outside. */
int oracle_locate(const oracle_cfg* cfg, int64_t np, const double* xyz, int32_t* cells)
{
    for (int64_t i = 0; i < np; ++i) {
        bool bad = false;
        Loc l;
        if (cfg->precision == 0) {
            Mesh<float> m = make_mesh<float>(cfg->n, cfg->origin, cfg->ending);
            l = locate<float>(m, (float)xyz[i], (float)xyz[np + i], (float)xyz[2 * np + i], bad);
        } else {
            Mesh<double> m = make_mesh<double>(cfg->n, cfg->origin, cfg->ending);
            l = locate<double>(m, xyz[i], xyz[np + i], xyz[2 * np + i], bad);
        }
        cells[i] = (bad || l.partitionI != 1) ? -1 : l.posI - 1;
    }
    return 0;
}

void oracle_pow0687(int64_t n, const double* x, double* y)
{
    for (int64_t i = 0; i < n; ++i) y[i] = st_pow0687(x[i]);
}

void oracle_pow0687f(int64_t n, const float* x, float* y)
{
    for (int64_t i = 0; i < n; ++i) y[i] = st_pow0687f(x[i]);
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"

namespace {

template <class P, class V>
int adjoint_run(const oracle_cfg* cfg, int64_t np, const double* xyz, const double* uvw,
                const double* d, const double* U, int T, double dt, const double* fscale,
                const double* cotangent, const double* target, int mean_limbs,
                double* mean_src, double* J_out, double* dalpha, double* dscale, double* dv0,
                int32_t* fz_cell, uint8_t* fz_bounce, int replay)
{
    if (cfg->n_substeps != 1 || cfg->drag != DRAG_SN_EXPLICIT) return -2;
    Params<P, V> pr = make_params<P, V>(cfg->n, cfg->origin, cfg->ending, cfg->mu_c, cfg->rho_c,
                                        cfg->rho_d, cfg->drag, 1, cfg->drag_multiplier,
                                        cfg->diameter_scale);
    const int64_t nC = pr.mesh.nCells;
    const P dtP = (P)dt;
    const V dtV = (V)dtP;
    const bool want_grad = dalpha || dscale || dv0;
    std::vector<Frozen> fz((size_t)T * np);
    if (replay)
        for (int64_t k = 0; k < (int64_t)T * np; ++k) fz[k] = Frozen{fz_cell[k], fz_bounce[k]};
    std::vector<V> vrec(want_grad ? (size_t)T * np * 3 : 0);
    /* fixed-point model of the mean source (constant scale over the T steps) */
    const int limbs = mean_limbs == 2 ? 2 : 1;
    const int64_t nbound = std::max<int64_t>(2, np * (int64_t)T);
    const int H = quant_headroom(limbs, nbound);
    int emax = EXP_NONE;
    for (int64_t i = 0; i < np; ++i) {  /* probe: largest deposit of the first step */
        P pos[3] = {(P)xyz[i], (P)xyz[np + i], (P)xyz[2 * np + i]};
        V vel[3] = {(V)uvw[i], (V)uvw[np + i], (V)uvw[2 * np + i]};
        Frozen f = replay ? fz[i] : Frozen{0, 0};
        StepLocal<V> o;
        V fs, fs_lo;
        split_factor<P, V>(fscale, 0, fs, fs_lo);
        if (!adj_forward_step<P, V>(pr, dtP, dtV, U, fs, fs_lo, pos, vel, (V)d[i], f,
                                    replay != 0, o))
            return -1;
        for (int c = 0; c < 3; ++c) {
            double dv = (double)o.dep[c];
            if (dv != 0.0 && std::isfinite(dv)) emax = std::max(emax, exp_of(dv));
        }
    }
    const int L = (emax == EXP_NONE) ? -H : emax - H;
    std::vector<int64_t> q1(limbs == 1 ? 3 * nC : 0, 0), hi(limbs == 2 ? 3 * nC : 0, 0);
    std::vector<uint64_t> lo(limbs == 2 ? 3 * nC : 0, 0);
    int64_t ovf = 0;
    for (int64_t i = 0; i < np; ++i) {
        P pos[3] = {(P)xyz[i], (P)xyz[np + i], (P)xyz[2 * np + i]};
        V vel[3] = {(V)uvw[i], (V)uvw[np + i], (V)uvw[2 * np + i]};
        for (int n = 0; n < T; ++n) {
            if (want_grad)
                for (int c = 0; c < 3; ++c) vrec[((size_t)n * np + i) * 3 + c] = vel[c];
            Frozen& f = fz[(size_t)n * np + i];
            StepLocal<V> o;
            V fs, fs_lo;
            split_factor<P, V>(fscale, n, fs, fs_lo);
            if (!adj_forward_step<P, V>(pr, dtP, dtV, U, fs, fs_lo, pos, vel, (V)d[i], f,
                                        replay != 0, o))
                return -1;
            for (int c = 0; c < 3; ++c) {
                double dv = (double)o.dep[c];
                if (dv == 0.0) continue;
                if (!std::isfinite(dv) || exp_of(dv) - L > H + QUANT_GROWTH_BITS) { ++ovf; continue; }
                int64_t q = std::llrint(ldexp2(dv, -L));
                const int64_t j = 3 * (int64_t)f.cell + c;
                if (limbs == 1) q1[j] = (int64_t)((uint64_t)q1[j] + (uint64_t)q);
                else { hi[j] += q >> 32; lo[j] += (uint64_t)q & 0xffffffffULL; }
            }
        }
    }
    std::vector<double> Sbar(3 * nC);
    for (int64_t j = 0; j < 3 * nC; ++j) {
        double v;
        if (limbs == 1) {
            v = (double)q1[j];
        } else {
            int64_t h = hi[j] + (int64_t)(lo[j] >> 32);
            v = (double)h * 4294967296.0 + (double)(lo[j] & 0xffffffffULL);
        }
        Sbar[j] = ldexp2(v, L) / (double)T;
    }
    if (mean_src) std::memcpy(mean_src, Sbar.data(), sizeof(double) * 3 * nC);
    double J = 0.0;
    std::vector<double> G(3 * nC, 0.0);
    for (int64_t j = 0; j < 3 * nC; ++j) {
        double yb;
        if (cotangent) {
            yb = cotangent[j];
        } else {
            const double r = Sbar[j] - (target ? target[j] : 0.0);
            J += r * r;
            yb = 2.0 * r;
        }
        G[j] = yb / (double)T;
    }
    if (J_out) *J_out = J;
    if (!replay && fz_cell)
        for (int64_t k = 0; k < (int64_t)T * np; ++k) {
            fz_cell[k] = fz[k].cell;
            fz_bounce[k] = fz[k].bounce;
        }
    if (!want_grad) return ovf ? 2 : 0;
    double da = 0.0, ds = 0.0;
    for (int64_t i = 0; i < np; ++i) {
        V a[3] = {(V)0, (V)0, (V)0};
        for (int n = T - 1; n >= 0; --n) {
            const Frozen& f = fz[(size_t)n * np + i];
            V vel[3];
            for (int c = 0; c < 3; ++c) vel[c] = vrec[((size_t)n * np + i) * 3 + c];
            V Gc[3];
            for (int c = 0; c < 3; ++c) Gc[c] = (V)G[3 * (int64_t)f.cell + c];
            V fs, fs_lo;
            split_factor<P, V>(fscale, n, fs, fs_lo);
            adj_reverse_step<P, V>(pr, dtP, dtV, U, fs, fs_lo, vel, (V)d[i], f, Gc, a, da, ds);
        }
        if (dv0)
            for (int c = 0; c < 3; ++c) dv0[c * np + i] = (double)a[c];
    }
    if (dalpha) *dalpha = da;
    if (dscale) *dscale = ds;
    return ovf ? 2 : 0;
}

}  // namespace

extern "C" {

/* Mean-source objective and its adjoint (SN drag, one substep), see adjoint_oracle.hpp.
 *  cotangent: dJ/dSbar [nCells][3], or NULL: J = sum (Sbar - target)^2 (target NULL = 0)
 *  mean_limbs: fixed-point model of the mean source (1 or 2 limbs, constant scale)
 *  fz_cell/fz_bounce [T][np]: frozen ownership, written (replay = 0) or read (replay = 1)
 * Returns 0, 2 (deposit out of range), -1 (parcel outside the mesh), -2 (unsupported). */
int oracle_adjoint(const oracle_cfg* cfg, int64_t np, const double* xyz, const double* uvw,
                   const double* d, const double* U, int T, double dt, const double* fscale,
                   const double* cotangent, const double* target, int mean_limbs,
                   double* mean_src, double* J_out, double* dalpha, double* dscale, double* dv0,
                   int32_t* fz_cell, uint8_t* fz_bounce, int replay)
{
    switch (cfg->precision) {
    case 1:
        return adjoint_run<double, float>(cfg, np, xyz, uvw, d, U, T, dt, fscale, cotangent,
                                          target, mean_limbs, mean_src, J_out, dalpha, dscale,
                                          dv0, fz_cell, fz_bounce, replay);
    case 2:
        return adjoint_run<double, double>(cfg, np, xyz, uvw, d, U, T, dt, fscale, cotangent,
                                           target, mean_limbs, mean_src, J_out, dalpha, dscale,
                                           dv0, fz_cell, fz_bounce, replay);
    default:
        return -2;
    }
}

}  // extern "C"

namespace {

template <class V>
int tet_run(const oracle_cfg* cfg, const TetMesh& mesh, int64_t np, double* xyz, double* uvw,
            const double* d, int32_t* cells, const double* U, int nsteps, double dt,
            const double* fscale, double* src_seq, double* src_quant, int32_t* scale_io,
            int64_t* stats, int64_t* hop_hist, int hop_limit)
{
    Params<double, V> pr = make_params<double, V>(cfg->n, cfg->origin, cfg->ending, cfg->mu_c,
                                                  cfg->rho_c, cfg->rho_d, cfg->drag,
                                                  cfg->n_substeps, cfg->drag_multiplier,
                                                  cfg->diameter_scale);
    const int64_t nC = mesh.nt;
    const double dtP = dt / (double)cfg->n_substeps;
    const V dtV = (V)dtP;
    const bool quant = src_quant != nullptr;
    const int limbs = cfg->quant_limbs == 2 ? 2 : 1;
    std::vector<int64_t> q1(limbs == 1 && quant ? 3 * nC : 0), hi(limbs == 2 && quant ? 3 * nC : 0);
    std::vector<uint64_t> lo(limbs == 2 && quant ? 3 * nC : 0);
    std::vector<double> seq(src_seq ? 3 * nC : 0);
    const int H = quant_headroom(limbs, std::max<int64_t>(2, np * (int64_t)cfg->n_substeps));
    int L = scale_io ? *scale_io : INT_MIN;
    int64_t lost = 0, ovf = 0;
    std::vector<double> P(3 * np);
    std::vector<V> Vv(3 * np), D(np);
    for (int64_t i = 0; i < np; ++i) {
        for (int c = 0; c < 3; ++c) {
            P[3 * i + c] = xyz[c * np + i];
            Vv[3 * i + c] = (V)uvw[c * np + i];
        }
        D[i] = (V)d[i];
    }
    for (int s = 0; s < nsteps; ++s) {
        V fs, fs_lo;
        split_factor<double, V>(fscale, s, fs, fs_lo);
        if (quant && L == INT_MIN) {
            Acc pa;
            pa.limbs = limbs; pa.L = 0; pa.H = 1 << 20;
            AccSink<V> sk(&pa, true);
            for (int64_t i = 0; i < np; ++i) {
                double x[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
                V v[3] = {Vv[3 * i], Vv[3 * i + 1], Vv[3 * i + 2]};
                int32_t c = cells[i];
                evolve_parcel_tet<V>(mesh, pr, dtP, dtV, U, fs, fs_lo, x, v, c, D[i], hop_limit,
                                     sk, nullptr);
            }
            L = (sk.emax == EXP_NONE) ? -H : sk.emax - H;
        }
        Acc acc;
        acc.limbs = limbs; acc.L = L; acc.H = H;
        if (src_seq) { std::fill(seq.begin(), seq.end(), 0.0); acc.seq = seq.data(); }
        if (quant) {
            if (limbs == 1) { std::fill(q1.begin(), q1.end(), 0); acc.q1 = q1.data(); }
            else {
                std::fill(hi.begin(), hi.end(), 0); std::fill(lo.begin(), lo.end(), 0);
                acc.hi = hi.data(); acc.lo = lo.data();
            }
        }
        AccSink<V> sk(&acc, quant);
        for (int64_t i = 0; i < np; ++i) {
            if (!evolve_parcel_tet<V>(mesh, pr, dtP, dtV, U, fs, fs_lo, &P[3 * i], &Vv[3 * i],
                                      cells[i], D[i], hop_limit, sk, hop_hist))
                ++lost;
        }
        ovf += sk.overflow;
        if (s == nsteps - 1 && quant) {
            for (int64_t j = 0; j < 3 * nC; ++j) {
                double v;
                if (limbs == 1) v = (double)q1[j];
                else {
                    int64_t h = hi[j] + (int64_t)(lo[j] >> 32);
                    v = (double)h * 4294967296.0 + (double)(lo[j] & 0xffffffffULL);
                }
                src_quant[j] = ldexp2(v, L);
            }
        }
        if (quant && sk.emax != EXP_NONE) L = sk.emax - H;
    }
    if (src_seq) std::memcpy(src_seq, seq.data(), sizeof(double) * 3 * nC);
    if (scale_io) *scale_io = L;
    for (int64_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c) {
            xyz[c * np + i] = P[3 * i + c];
            uvw[c * np + i] = (double)Vv[3 * i + c];
        }
    if (stats) { stats[0] = lost; stats[1] = ovf; stats[2] = H; }
    return (lost ? 1 : 0) | (ovf ? 2 : 0);
}

}  // namespace

extern "C" {

/* Steps on a tetrahedral mesh (face walk).  cells [np]: tet of each parcel, in/out.
 * box from cfg->origin/ending; precision 1 (mixed) or 2 (FP64).  hop_hist[8]: histogram
 * of walk lengths (hops per substep, last bin 7+), or NULL.  Returns as oracle_run. */
int oracle_tet_run(const oracle_cfg* cfg, int64_t nv, const double* verts, int64_t nt,
                   const int32_t* tets, const int32_t* nbr, int64_t np, double* xyz,
                   double* uvw, const double* d, int32_t* cells, const double* U, int nsteps,
                   double dt, const double* fscale, double* src_seq, double* src_quant,
                   int32_t* scale_io, int64_t* stats, int64_t* hop_hist, int hop_limit)
{
    std::vector<int32_t> ct(4 * nt), cn(4 * nt);
    canonical_tets(nt, tets, nbr, ct.data(), cn.data());
    TetMesh m;
    m.nv = nv; m.nt = nt; m.verts = verts; m.tets = ct.data(); m.nbr = cn.data();
    for (int a = 0; a < 3; ++a) { m.origin[a] = cfg->origin[a]; m.ending[a] = cfg->ending[a]; }
    if (cfg->precision == 1)
        return tet_run<float>(cfg, m, np, xyz, uvw, d, cells, U, nsteps, dt, fscale, src_seq,
                              src_quant, scale_io, stats, hop_hist, hop_limit);
    if (cfg->precision == 2)
        return tet_run<double>(cfg, m, np, xyz, uvw, d, cells, U, nsteps, dt, fscale, src_seq,
                               src_quant, scale_io, stats, hop_hist, hop_limit);
    return -2;
}

/* Parcels of st_init_parcels (the shared generator of st_init.h): positions rounded to
 * the position precision (pbytes 4 or 8) and returned as doubles, [3][n]; diameters in
 * double (the library rounds them to the velocity precision). */
void oracle_init_parcels(int pbytes, uint64_t seed, int cloud, int nclouds, int64_t n,
                         const int32_t N[3], const double origin[3], const double ending[3],
                         double d_min, double d_max, double* xyz, double* d)
{
    for (int64_t j = 0; j < n; ++j) {
        if (pbytes == 4) {
            float p[3];
            st_init_parcel<float>(seed, cloud, nclouds, (uint64_t)j, N, origin, ending, p, d[j],
                                  d_min, d_max);
            for (int a = 0; a < 3; ++a) xyz[a * n + j] = p[a];
        } else {
            double p[3];
            st_init_parcel<double>(seed, cloud, nclouds, (uint64_t)j, N, origin, ending, p, d[j],
                                   d_min, d_max);
            for (int a = 0; a < 3; ++a) xyz[a * n + j] = p[a];
        }
    }
}

/* Hilbert curve point of each index (3 x bits bits) */
void oracle_hilbert3(int64_t n, const uint64_t* h, int bits, uint32_t* p)
{
    for (int64_t i = 0; i < n; ++i) st_hilbert3(h[i], bits, p + 3 * i);
}

/* Walk from start[i] to the tet containing xyz[:, i]; status[i] as WALK_*. */
int oracle_tet_locate(int64_t nv, const double* verts, int64_t nt, const int32_t* tets,
                      const int32_t* nbr, int64_t np, const double* xyz, const int32_t* start,
                      int32_t* cells, int32_t* status, int hop_limit)
{
    std::vector<int32_t> ct(4 * nt), cn(4 * nt);
    canonical_tets(nt, tets, nbr, ct.data(), cn.data());
    TetMesh m;
    m.nv = nv; m.nt = nt; m.verts = verts; m.tets = ct.data(); m.nbr = cn.data();
    for (int64_t i = 0; i < np; ++i) {
        double x[3] = {xyz[i], xyz[np + i], xyz[2 * np + i]};
        int st = 0, hops = 0;
        cells[i] = tet_walk(m, start[i], x, hop_limit, st, hops);
        status[i] = st;
    }
    return 0;
}

}  // extern "C"
