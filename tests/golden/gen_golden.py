"""Generates the golden fixtures in tests/golden/*.npz.

An independent, line-by-line restatement of the reference's parcel step in numpy float32
scalars (Julia Float32 arithmetic is IEEE binary32 without fma contraction, and so are
numpy float32 scalar operations), and of the library's mixed-precision and all-FP64 modes
in Python floats (binary64) and numpy float32 scalars.  It deliberately shares no code with
the C++ oracle, so agreement between the two is a cross-check of both restatements.

Fixtures: ref_stokes_fp32, sn_fp32, sn_bench_fp32 (FP32 reference mode, fluid factor 1);
sn_mixed, sn_sub3_mixed, stokes_mixed, sn_bench_mixed, stokes_wide_mixed, sn_sub3_fp64,
stokes_fp64, stokes_wide_fp64 (binary64 positions, a time-varying fluid factor per step in
`fscale`, the mode in `precision`).  Each
holds the last step's source twice: `src_f64`, the FP64 sum of the deposits in parcel order,
and `src_quant`, the library's deterministic fixed-point source (fixed_point_source).

Reference file (A:): run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
  locate_ijk / locate ........................ A:663-697
  update! (CPU, '+=') / update_at_boundary! .. A:703-708, A:731-736
  evolve_particle! ........................... A:1271-1365
  CPU executor loop, Δt/nSteps ............... A:818-823, A:1260
  Mesh construction (Float64 -> Float32) ..... A:237-268

The Schiller-Naumann drag is project-defined (the reference only has Stokes drag); its
power functions follow the same algorithms as scale-track_b200/csrc/st_pow.h, restated here
in Python floats (double) and numpy float32 scalars with an exact-rational fma (single).

Tet fixtures (tests/golden/tet/*.npz): the library's face walk on a jittered tet mesh with
the mixed and FP64 step, restated the same way (TetMesh, evolve_parcel_tet).

Run:  python tests/golden/gen_golden.py      (rewrites the .npz files next to this script)
"""
import math
import os
import struct
from fractions import Fraction

import numpy as np

F = np.float32
HERE = os.path.dirname(os.path.abspath(__file__))


# ----------------------------------------------------------------------------- power helper
def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _dbl(b):
    return struct.unpack("<d", struct.pack("<Q", b))[0]


def _pow2i(k):
    return _dbl((k + 1023) << 52)


def _log_pos(x):
    LN2 = 0.69314718055994530942
    SQRT2 = 1.41421356237309504880
    e = 0
    if x < 2.2250738585072014e-308:
        x = x * 18014398509481984.0
        e = -54
    b = _bits(x)
    e += ((b >> 52) & 0x7FF) - 1023
    m = _dbl((b & 0x000FFFFFFFFFFFFF) | 0x3FF0000000000000)
    if m > SQRT2:
        m = m * 0.5
        e += 1
    s = (m - 1.0) / (m + 1.0)
    z = s * s
    p = 1.0 / 23.0
    for c in (21.0, 19.0, 17.0, 15.0, 13.0, 11.0, 9.0, 7.0, 5.0, 3.0):
        p = p * z + 1.0 / c
    p = p * z + 1.0
    return float(e) * LN2 + (2.0 * s) * p


def _exp_small(y):
    LN2 = 0.69314718055994530942
    INV_LN2 = 1.44269504088896340736
    t = y * INV_LN2
    k = int(t + 0.5) if t >= 0.0 else -int(-t + 0.5)
    r = y - float(k) * LN2
    p = 1.0 / 87178291200.0
    for c in (6227020800.0, 479001600.0, 39916800.0, 3628800.0, 362880.0, 40320.0, 5040.0,
              720.0, 120.0, 24.0, 6.0):
        p = p * r + 1.0 / c
    p = p * r + 0.5
    p = p * r + 1.0
    p = p * r + 1.0
    k1 = int(k / 2)
    k2 = k - k1
    return (p * _pow2i(k1)) * _pow2i(k2)


def pow0687(x):
    x = float(x)
    if not (x > 0.0):
        return x if x != x else 0.0
    if x > 1.0e300:
        return x
    return _exp_small(0.687 * _log_pos(x))


def _fbits(x):
    return int(np.array([x], dtype=np.float32).view(np.uint32)[0])


def _ffrom(b):
    return np.array([b], dtype=np.uint32).view(np.float32)[0]


def fmaf(a, b, c):
    """Single-precision fused multiply-add, rounded once: a*b + c is formed exactly as a
    rational number and rounded to the nearest binary32 value (ties to even)."""
    v = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    if v == 0:
        return F(0)
    sign = -1 if v < 0 else 1
    v = abs(v)
    ex = v.numerator.bit_length() - v.denominator.bit_length()
    if Fraction(2) ** ex > v:
        ex -= 1                                   # now 2^ex <= v < 2^(ex+1)
    quantum = Fraction(2) ** (max(ex, -126) - 23)
    q = v / quantum
    n = q.numerator // q.denominator
    rem = q - n
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and n % 2 == 1):
        n += 1
    return F(sign * float(n * quantum))          # exact: n * quantum is a binary32 value


# coefficients of st_pow0687f (printed by scale-track_b200/csrc/pow_coeffs.py)
_PT = [float.fromhex(h) for h in ("0x1p+0", "0x1.5fbe76p-1", "-0x1.b862bep-4", "0x1.817e2ap-5",
                                  "-0x1.bd5c3ap-6", "0x1.2657a8p-6", "-0x1.b6bb7ep-7",
                                  "0x1.68372ap-7", "-0x1.921f0ep-8")]
_PR = [float.fromhex(h) for h in ("0x1p+0", "0x1.6b689cp-11", "0x1.01f20ep-22",
                                  "0x1.e8030ap-35", "0x1.5cea7ap-47", "0x1.6dafdep-60",
                                  "0x1.08638ep-72")]


def pow0687f(x):
    """Single-precision x^0.687 (same algorithm as st_pow0687f): x = 2^e m, t = m - 1,
    687 e = 1000 k + r; (1+t)^0.687 and 2^(r/1000) by Horner with fma, times 2^k."""
    x = F(x)
    if not (x > F(0)):
        return x if x != x else F(0)
    b = _fbits(x)
    if (b >> 23) == 0xFF:
        return x
    e = 0
    if (b >> 23) == 0:
        x = F(x * F(16777216.0))
        e = -24
        b = _fbits(x)
    e += ((b >> 23) & 0xFF) - 127
    m = _ffrom((b & 0x007FFFFF) | 0x3F800000)
    if m > F(1.41421356):
        m = F(m * F(0.5))
        e += 1
    t = F(m - F(1))
    p = F(_PT[8])
    for c in reversed(_PT[:8]):
        p = fmaf(p, t, F(c))
    y = 687 * e
    k = y // 1000                                 # floor division
    r = F(y - 1000 * k)
    q = F(_PR[6])
    for c in reversed(_PR[:6]):
        q = fmaf(q, r, F(c))
    return F(F(p * q) * _ffrom((k + 127) << 23))


# --------------------------------------------------------- the deterministic source model
def fixed_point_source(step_logs, ncells, npcl, nsub, limbs):
    """The library's deterministic source of the last step (project-defined; the reference
    adds Float32 atomics), from each step's deposits [(1-based cell, [three components])]:
    a component v != 0 becomes round(v 2^-L) (ties to even) and the integers are summed per
    cell, so the order of the deposits does not matter; the source is the sum times 2^L.
    The scale of a step is L = emax - H, emax the largest frexp exponent of the previous
    step's deposits (of the same step's for the first one, which the library finds by a
    read-only pass), H = 54 - nb headroom bits for one 64-bit limb (nb: smallest with
    2^nb >= parcels x substeps, at least 1 and 2 deposits) or 54 for two limbs."""
    nbound = max(2, npcl * nsub)
    nb = 1
    while nb < 62 and (1 << nb) < nbound:
        nb += 1
    H = 62 - 8 - nb if limbs == 1 else 62 - 8

    def emax(log):
        es = [math.frexp(v)[1] for _, comps in log for v in comps if v != 0.0]
        return max(es) if es else None

    e1 = emax(step_logs[0])
    L = e1 - H if e1 is not None else -H
    for k, log in enumerate(step_logs):
        Q = [[0, 0, 0] for _ in range(ncells)]
        for cell, comps in log:
            for c, v in enumerate(comps):
                if v == 0.0:
                    continue
                assert math.frexp(v)[1] - L <= H + 8, "deposit outside the fixed-point range"
                Q[cell - 1][c] += round(math.ldexp(v, -L))
        if k == len(step_logs) - 1:
            return np.array([[math.ldexp(float(q), L) for q in row] for row in Q])
        e = emax(log)
        if e is not None:
            L = e - H


# ----------------------------------------------------------------------------- the step
class Mesh:
    """construct_mesh (A:237-268) with decomposition (1,1,1)."""

    def __init__(self, n, origin, ending):
        self.N = [int(v) for v in n]
        self.origin = [F(o) for o in origin]
        self.rD = []
        for a in range(3):
            L = float(ending[a]) - float(origin[a])
            D = L / float(n[a])
            self.rD.append(F(1.0 / D))
        self.NxNy = self.N[0] * self.N[1]


def floor_label(v):
    f = np.floor(v)
    assert -2.0 ** 31 <= float(f) < 2.0 ** 31
    return int(f)


def _divrem(a, b):
    q = abs(a) // b
    q = q if a >= 0 else -q
    return q, a - q * b


def locate(m, x, y, z):
    I = floor_label(F(x - m.origin[0]) * m.rD[0])
    J = floor_label(F(y - m.origin[1]) * m.rD[1])
    K = floor_label(F(z - m.origin[2]) * m.rD[2])
    iP, iL = _divrem(I, m.N[0])
    jP, jL = _divrem(J, m.N[1])
    kP, kL = _divrem(K, m.N[2])
    part = abs(kP) + abs(jP) + abs(iP) + 1
    pos = abs(kL) * m.NxNy + abs(jL) * m.N[0] + abs(iL) + 1
    return I, J, K, pos, part


def evolve_particle(m, prm, X, Y, Z, U, V, W, dIn, Ucell, fs, dt, nsteps, UTrans32, UTrans64,
                    log):
    mu, rho_d, rr, rnu, drag = prm["mu"], prm["rho_d"], prm["rr"], prm["rnu"], prm["drag"]
    d = F(dIn * F(1.0))
    mB = F(F(F(rr * F(math.pi)) * F(F(d * d) * d)) / F(6))
    pos = [X, Y, Z]
    vel = [U, V, W]
    posNew = list(pos)
    velNew = list(vel)
    I, J, K, posI, partI = locate(m, *pos)
    assert partI == 1
    uc = [F(Ucell[posI - 1][c] * fs) for c in range(3)]
    state0 = list(vel)
    f = F(F(F(F(18) * mu) * dt) / F(rho_d * F(d * d)))

    def deposit(cell, s0, vn):
        deps = []
        for c in range(3):
            dep = F(mB * F(s0[c] - vn[c]))
            UTrans32[cell - 1][c] = F(UTrans32[cell - 1][c] + dep)
            UTrans64[cell - 1][c] = UTrans64[cell - 1][c] + float(dep)
            deps.append(float(dep))
        log.append((cell, deps))

    for t in range(1, nsteps + 1):
        if drag == 0:
            for c in range(3):
                velNew[c] = F(F(vel[c] + F(f * uc[c])) / F(F(1) + f))
        else:
            du = [F(uc[c] - vel[c]) for c in range(3)]
            mag = F(np.sqrt(F(F(F(du[0] * du[0]) + F(du[1] * du[1])) + F(du[2] * du[2]))))
            Re = F(F(mag * d) * rnu)
            pw = pow0687f(Re)
            g = F(f * F(F(1) + F(F(0.15) * pw)))
            for c in range(3):
                velNew[c] = F(vel[c] + F(g * du[c]))
        for c in range(3):
            posNew[c] = F(pos[c] + F(velNew[c] * dt))
        I, J, K, posNewI, partNewI = locate(m, *posNew)
        if posNewI != posI or partNewI != partI:
            b = [I < 0 or I >= m.N[0], J < 0 or J >= m.N[1], K < 0 or K >= m.N[2]]
            for c in range(3):
                if b[c]:
                    posNew[c] = pos[c]
                    velNew[c] = F(-vel[c])
                    state0[c] = F(state0[c] - F(F(2) * vel[c]))
            if any(b):
                I, J, K, posNewI, partNewI = locate(m, *posNew)
            if t != nsteps and posNewI != posI:
                deposit(posI, state0, velNew)
                state0 = list(velNew)
                uc = [F(Ucell[posNewI - 1][c] * fs) for c in range(3)]
                posI = posNewI
        vel = list(velNew)
        pos = list(posNew)
    deposit(posI, state0, velNew)
    return posNew, velNew


def run_case(n, origin, ending, mu_c, rho_c, rho_d, drag, nsub, xyz, uvw, d, Ucell, dt, nsteps):
    m = Mesh(n, origin, ending)
    prm = dict(mu=F(mu_c), rho_d=F(rho_d), rr=F(rho_d / rho_c), rnu=F(rho_c / mu_c), drag=drag)
    npcl = d.shape[0]
    X = [F(v) for v in xyz[0]]
    Y = [F(v) for v in xyz[1]]
    Z = [F(v) for v in xyz[2]]
    U = [F(v) for v in uvw[0]]
    V = [F(v) for v in uvw[1]]
    W = [F(v) for v in uvw[2]]
    D = [F(v) for v in d]
    Uc = [[F(v) for v in row] for row in Ucell]
    dtF = F(F(dt) / F(nsub))
    ncells = n[0] * n[1] * n[2]
    logs = []
    for s in range(nsteps):
        UT32 = [[F(0), F(0), F(0)] for _ in range(ncells)]
        UT64 = [[0.0, 0.0, 0.0] for _ in range(ncells)]
        logs.append([])
        for i in range(npcl):
            p, v = evolve_particle(m, prm, X[i], Y[i], Z[i], U[i], V[i], W[i], D[i], Uc, F(1),
                                   dtF, nsub, UT32, UT64, logs[-1])
            X[i], Y[i], Z[i] = p
            U[i], V[i], W[i] = v
    cells = []
    for i in range(npcl):
        _, _, _, pos, part = locate(m, X[i], Y[i], Z[i])
        cells.append(pos - 1 if part == 1 else -1)
    return dict(
        xyz=np.array([X, Y, Z], dtype=np.float32),
        uvw=np.array([U, V, W], dtype=np.float32),
        cells=np.array(cells, dtype=np.int32),
        src_f32=np.array(UT32, dtype=np.float32),
        src_f64=np.array(UT64, dtype=np.float64),
        src_quant=fixed_point_source(logs, ncells, npcl, nsub, limbs=1),
    )


# ------------------------------------------------- mixed precision and all-FP64 (P = double)
# Project-defined modes of the library (the reference computes in Float32 only), restated
# from their definitions: positions, the substep for positions and the cell location in
# binary64 (Python floats); in mixed precision drag, velocity and deposit in binary32 with the
# compensated slip u_c - v = fma(U, fs_hi, -v) + U fs_lo (fs = fs_hi + fs_lo, the step's FP64
# fluid factor split into a float and its remainder) and the increment-tracked deposit
# D = state0 - v (each substep subtracts its velocity increment, a bounced component keeps
# its D, a deposit is m/rho_c D); all-FP64 follows the reference's form in binary64.

class Mesh64:
    """construct_mesh (A:237-268) with the spacing kept in binary64 (P = double)."""

    def __init__(self, n, origin, ending):
        self.N = [int(v) for v in n]
        self.origin = [float(o) for o in origin]
        self.rD = [1.0 / ((float(ending[a]) - float(origin[a])) / float(n[a]))
                   for a in range(3)]
        self.NxNy = self.N[0] * self.N[1]


def locate64(m, x, y, z):
    lab = []
    for a, v in enumerate((x, y, z)):
        f = math.floor((v - m.origin[a]) * m.rD[a])
        assert -2.0 ** 31 <= f < 2.0 ** 31
        lab.append(int(f))
    I, J, K = lab
    iP, iL = _divrem(I, m.N[0])
    jP, jL = _divrem(J, m.N[1])
    kP, kL = _divrem(K, m.N[2])
    part = abs(kP) + abs(jP) + abs(iP) + 1
    pos = abs(kL) * m.NxNy + abs(jL) * m.N[0] + abs(iL) + 1
    return I, J, K, pos, part


def _walls(m, I, J, K):
    return [I < 0 or I >= m.N[0], J < 0 or J >= m.N[1], K < 0 or K >= m.N[2]]


def evolve_particle_mixed(m, prm, pos, vel, dIn, Ucell, fs_hi, fs_lo, dtP, dtV, nsteps,
                          UTrans64, log):
    """evolve_particle! (A:1271-1365) with binary64 positions and binary32 drag/velocity."""
    mu, rho_d, rr, rnu, drag = prm["mu"], prm["rho_d"], prm["rr"], prm["rnu"], prm["drag"]
    d = F(dIn * F(1.0))
    mB = F(F(F(rr * F(math.pi)) * F(F(d * d) * d)) / F(6))
    f = F(F(F(F(F(18) * mu) * dtV) / F(rho_d * F(d * d))) * F(1.0))
    pos, vel = list(pos), list(vel)
    _, _, _, posI, part = locate64(m, *pos)
    assert part == 1
    Ur = [F(Ucell[posI - 1][c]) for c in range(3)]
    D = [F(0), F(0), F(0)]

    def slip(c):
        return F(fmaf(Ur[c], fs_hi, F(-vel[c])) + F(Ur[c] * fs_lo))

    def deposit(cell):
        deps = [float(F(mB * D[c])) for c in range(3)]
        for c in range(3):
            UTrans64[cell - 1][c] = UTrans64[cell - 1][c] + deps[c]
        log.append((cell, deps))

    for t in range(1, nsteps + 1):
        inc = [F(0)] * 3
        if drag == 0:
            inc = [F(F(f * slip(c)) / F(F(1) + f)) for c in range(3)]
        else:
            du = [slip(c) for c in range(3)]
            mag = F(np.sqrt(F(F(F(du[0] * du[0]) + F(du[1] * du[1])) + F(du[2] * du[2]))))
            Re = F(F(mag * d) * rnu)
            g = F(f * F(F(1) + F(F(0.15) * pow0687f(Re))))
            inc = [F(g * du[c]) for c in range(3)]
        velNew = [F(vel[c] + inc[c]) for c in range(3)]
        posNew = [pos[c] + float(velNew[c]) * dtP for c in range(3)]
        I, J, K, posNewI, partNew = locate64(m, *posNew)
        b = [False, False, False]
        if posNewI != posI or partNew != 1:
            b = _walls(m, I, J, K)
            for c in range(3):
                if b[c]:
                    posNew[c] = pos[c]
                    velNew[c] = F(-vel[c])
            if any(b):
                I, J, K, posNewI, partNew = locate64(m, *posNew)
        for c in range(3):
            if not b[c]:
                D[c] = F(D[c] - inc[c])
        if t != nsteps and posNewI != posI:
            deposit(posI)
            D = [F(0), F(0), F(0)]
            Ur = [F(Ucell[posNewI - 1][c]) for c in range(3)]
            posI = posNewI
        vel, pos = velNew, posNew
    deposit(posI)
    return pos, vel


def evolve_particle_fp64(m, prm, pos, vel, dIn, Ucell, fs, dtP, dtV, nsteps, UTrans64, log):
    """evolve_particle! (A:1271-1365) in binary64 throughout, the reference's form."""
    mu, rho_d, rr, rnu, drag = prm["mu"], prm["rho_d"], prm["rr"], prm["rnu"], prm["drag"]
    d = dIn * 1.0
    mB = ((rr * math.pi) * ((d * d) * d)) / 6.0
    f = ((((18.0 * mu) * dtV) / (rho_d * (d * d)))) * 1.0
    pos, vel = list(pos), list(vel)
    _, _, _, posI, part = locate64(m, *pos)
    assert part == 1
    Ur = [float(Ucell[posI - 1][c]) for c in range(3)]
    state0 = list(vel)

    def deposit(cell, vn):
        deps = [mB * (state0[c] - vn[c]) for c in range(3)]
        for c in range(3):
            UTrans64[cell - 1][c] = UTrans64[cell - 1][c] + deps[c]
        log.append((cell, deps))

    for t in range(1, nsteps + 1):
        if drag == 0:
            velNew = [(vel[c] + f * (Ur[c] * fs)) / (1.0 + f) for c in range(3)]
        else:
            du = [Ur[c] * fs - vel[c] for c in range(3)]
            mag = math.sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2])
            Re = (mag * d) * rnu
            g = f * (1.0 + 0.15 * pow0687(Re))
            velNew = [vel[c] + g * du[c] for c in range(3)]
        posNew = [pos[c] + velNew[c] * dtP for c in range(3)]
        I, J, K, posNewI, partNew = locate64(m, *posNew)
        if posNewI != posI or partNew != 1:
            b = _walls(m, I, J, K)
            for c in range(3):
                if b[c]:
                    posNew[c] = pos[c]
                    velNew[c] = -vel[c]
                    state0[c] = state0[c] - 2.0 * vel[c]
            if any(b):
                I, J, K, posNewI, partNew = locate64(m, *posNew)
        if t != nsteps and posNewI != posI:
            deposit(posI, velNew)
            state0 = list(velNew)
            Ur = [float(Ucell[posNewI - 1][c]) for c in range(3)]
            posI = posNewI
        vel, pos = velNew, posNew
    deposit(posI, velNew)
    return pos, vel


def run_case_p64(n, origin, ending, mu_c, rho_c, rho_d, drag, nsub, xyz, uvw, d, Ucell, dt,
                 nsteps, fscale, precision):
    """The CPU executor loop (A:818-823) in mixed precision or all-FP64; step s uses the
    fluid factor fscale[s] on the cell velocities."""
    m = Mesh64(n, origin, ending)
    mixed = precision == "mixed"
    V = F if mixed else float
    prm = dict(mu=V(mu_c), rho_d=V(rho_d), rr=V(rho_d / rho_c), rnu=V(rho_c / mu_c), drag=drag)
    npcl = d.shape[0]
    P = [[float(v) for v in xyz[a]] for a in range(3)]
    W = [[V(v) for v in uvw[a]] for a in range(3)]
    D = [V(v) for v in d]
    Uc = [[V(v) for v in row] for row in Ucell]
    dtP = float(dt) / float(nsub)
    dtV = V(dtP)
    ncells = n[0] * n[1] * n[2]
    logs = []
    for s in range(nsteps):
        UT64 = [[0.0, 0.0, 0.0] for _ in range(ncells)]
        logs.append([])
        fs = float(fscale[s])
        for i in range(npcl):
            pos = [P[0][i], P[1][i], P[2][i]]
            vel = [W[0][i], W[1][i], W[2][i]]
            if mixed:
                hi = F(fs)
                lo = F(fs - float(hi))
                p, v = evolve_particle_mixed(m, prm, pos, vel, D[i], Uc, hi, lo, dtP, dtV, nsub,
                                             UT64, logs[-1])
            else:
                p, v = evolve_particle_fp64(m, prm, pos, vel, D[i], Uc, fs, dtP, dtV, nsub,
                                            UT64, logs[-1])
            for a in range(3):
                P[a][i] = p[a]
                W[a][i] = v[a]
    cells = []
    for i in range(npcl):
        _, _, _, pos, part = locate64(m, P[0][i], P[1][i], P[2][i])
        cells.append(pos - 1 if part == 1 else -1)
    return dict(
        xyz=np.array(P, dtype=np.float64),
        uvw=np.array(W, dtype=np.float32 if mixed else np.float64),
        cells=np.array(cells, dtype=np.int32),
        src_f64=np.array(UT64, dtype=np.float64),
        src_quant=fixed_point_source(logs, ncells, npcl, nsub, limbs=1 if mixed else 2),
    )


def make_inputs64(seed, n, npcl, ending, dmin, dmax, precision, v0_random=True, dlog=False):
    """Inputs of the binary64-position cases: positions uniform in the box as binary64 values
    (not float32-representable), hand-placed parcels on walls, faces and one ulp inside the
    upper walls; velocities, diameters and cell velocities in the velocity precision."""
    rng = np.random.default_rng(seed)
    vt = np.float32 if precision == "mixed" else np.float64
    xyz = rng.random((3, npcl)) * float(ending)
    h = float(ending) / n
    top = np.nextafter(float(ending), 0.0)
    special = [(0.0, 0.5 * ending, 0.5 * ending), (top, 0.5 * ending, 0.5 * ending),
               (0.5 * ending, top, 0.5 * ending), (0.5 * ending, 0.5 * ending, top),
               (h, h, h), (2 * h, 0.5 * ending, 3 * h), (0.0, 0.0, 0.0)]
    for k, s3 in enumerate(special):
        xyz[:, k] = s3
    uvw = (rng.random((3, npcl)) * 2.0 - 1.0) if v0_random else np.zeros((3, npcl))
    uvw[:, :7] = np.array([[-0.9, 0.1, 0.2], [0.8, -0.3, 0.1], [0.1, -0.95, 0.0],
                           [0.0, 0.2, 0.9], [-0.5, -0.5, -0.5], [0.3, 0.0, -0.4],
                           [-1.0, -1.0, -1.0]]).T
    uvw = uvw.astype(vt)
    if dlog:   # log-uniform: deposits over many decades, rounded at the fixed-point scale
        d = np.exp(rng.random(npcl) * (math.log(dmax) - math.log(dmin)) + math.log(dmin))
        d = d.astype(vt)
    else:
        d = (rng.random(npcl) * (dmax - dmin) + dmin).astype(vt)
    Ucell = (rng.random((n ** 3, 3)) * 2.0 - 1.0).astype(vt)
    return xyz, uvw, d, Ucell


def fluid_factors(nsteps):
    """A time-varying fluid factor per step whose values are not binary32-representable (so
    the low part of the split is not zero)."""
    return np.array([1.0 + 0.2 * math.sin(0.37 * (s + 1) + 0.3) for s in range(nsteps)])


def make_inputs(seed, n, npcl, ending, dmin, dmax, v0_random=False, wall_cases=True):
    """Parcels uniform in the box (as init! does, A:518-525), diameters U[dmin, dmax),
    random cell velocity in [-1, 1) (the REPL test block, A:1645-1650), plus hand-placed
    parcels at walls, on faces and at the origin."""
    rng = np.random.default_rng(seed)
    xyz = rng.random((3, npcl)).astype(np.float32) * np.float32(ending)
    if wall_cases:
        f = 1.0 / n
        special = [  # fractions of the box edge: walls, exact faces, the origin
            (0.0, 0.5, 0.5), (0.99999, 0.5, 0.5), (0.5, 1e-4, 0.5), (0.5, 0.5, 0.9999),
            (f, f, f), (2 * f, 0.5, 3 * f), (0.0, 0.0, 0.0),
        ]
        for k, s in enumerate(special):
            xyz[:, k] = np.array(s, dtype=np.float32) * np.float32(ending)
    uvw = np.zeros((3, npcl), dtype=np.float32)
    if v0_random:
        uvw = (rng.random((3, npcl)) * 2.0 - 1.0).astype(np.float32)
    uvw[:, :7] = np.array([[-0.9, 0.1, 0.2], [0.8, -0.3, 0.1], [0.1, -0.95, 0.0],
                           [0.0, 0.2, 0.9], [-0.5, -0.5, -0.5], [0.3, 0.0, -0.4],
                           [-1.0, -1.0, -1.0]], dtype=np.float32).T
    d = (rng.random(npcl) * (dmax - dmin) + dmin).astype(np.float32)
    ncells = n ** 3
    Ucell = (rng.random((ncells, 3)) * 2.0 - 1.0).astype(np.float32)
    return xyz, uvw, d, Ucell


CASES = {
    # reference physics (setup.jl: μᶜ=1e-3, ρᶜ=1e3, ρᵈ=1, d in [5e-3, 1e-2)), Stokes implicit,
    # 10 substeps, a large Δt so that parcels cross faces and hit walls
    "ref_stokes_fp32": dict(seed=11, n=8, npcl=96, ending=1.0, dmin=5e-3, dmax=1e-2,
                            mu_c=1e-3, rho_c=1e3, rho_d=1.0, drag=0, nsub=10, dt=0.6, nsteps=3),
    # same geometry, Schiller-Naumann explicit drag, one substep
    "sn_fp32": dict(seed=12, n=8, npcl=96, ending=1.0, dmin=5e-3, dmax=1e-2,
                    mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=1, nsub=1, dt=0.05, nsteps=4,
                    v0_random=True),
    # the benchmark's physical constants on a small box
    "sn_bench_fp32": dict(seed=13, n=6, npcl=64, ending=0.01, dmin=1e-5, dmax=4e-5,
                          mu_c=1.8e-5, rho_c=1.2, rho_d=1000.0, drag=1, nsub=1, dt=4e-4,
                          nsteps=3),
}

# binary64-position cases: (name, precision, case); every one has a time-varying fluid factor
CASES64 = {
    # Schiller-Naumann, one substep, reference-physics box with dense parcels
    "sn_mixed": dict(precision="mixed", seed=21, n=8, npcl=96, ending=1.0, dmin=5e-3, dmax=1e-2,
                     mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=1, nsub=1, dt=0.05, nsteps=4),
    # Schiller-Naumann, three substeps: intermediate deposits at cell crossings
    "sn_sub3_mixed": dict(precision="mixed", seed=22, n=8, npcl=96, ending=1.0, dmin=5e-3,
                          dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=1, nsub=3,
                          dt=0.15, nsteps=3),
    # Stokes implicit, ten substeps, the reference's physics and a large step (walls, faces)
    "stokes_mixed": dict(precision="mixed", seed=23, n=8, npcl=96, ending=1.0, dmin=5e-3,
                         dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1.0, drag=0, nsub=10, dt=0.6,
                         nsteps=3),
    # the benchmark's physical constants on a small box
    "sn_bench_mixed": dict(precision="mixed", seed=24, n=6, npcl=64, ending=0.01, dmin=1e-5,
                           dmax=4e-5, mu_c=1.8e-5, rho_c=1.2, rho_d=1000.0, drag=1, nsub=1,
                           dt=4e-4, nsteps=3),
    "sn_sub3_fp64": dict(precision="fp64", seed=25, n=8, npcl=96, ending=1.0, dmin=5e-3,
                         dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=1, nsub=3,
                         dt=0.15, nsteps=3),
    "stokes_fp64": dict(precision="fp64", seed=26, n=8, npcl=96, ending=1.0, dmin=5e-3,
                        dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1.0, drag=0, nsub=10, dt=0.6,
                        nsteps=3),
    # diameters log-uniform over four decades: deposit magnitudes span about 2^40, so the
    # small parcels' deposits are rounded at the fixed-point scale (one limb and two)
    "stokes_wide_mixed": dict(precision="mixed", seed=27, n=8, npcl=96, ending=1.0, dmin=1e-6,
                              dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=0, nsub=2,
                              dt=0.1, nsteps=3, dlog=True),
    "stokes_wide_fp64": dict(precision="fp64", seed=28, n=8, npcl=96, ending=1.0, dmin=1e-6,
                             dmax=1e-2, mu_c=1e-3, rho_c=1e3, rho_d=1000.0, drag=0, nsub=2,
                             dt=0.1, nsteps=3, dlog=True),
}


def _cells0(c, xyz):
    m = Mesh([c["n"]] * 3, [0.0] * 3, [c["ending"]] * 3)
    return np.array([locate(m, *xyz[:, i])[3] - 1 for i in range(xyz.shape[1])])


def _cells0_64(c, xyz):
    m = Mesh64([c["n"]] * 3, [0.0] * 3, [c["ending"]] * 3)
    return np.array([locate64(m, *xyz[:, i])[3] - 1 for i in range(xyz.shape[1])])


# ------------------------------------------------ tetrahedral meshes (project-defined walk)
# The library's face walk on a conforming tet mesh, restated from its definition: each tet's
# vertex ids sorted increasingly (neighbours permuted with them); face f has the other three
# vertices (p, q, r) in increasing order, n = (q - p) x (r - p), negated when n.(v_f - p) > 0,
# c = n.p and s_f(x) = n.x - c in binary64; a walk moves across the face with the largest
# positive s_f (ties to the lowest f) until no s_f is positive.  The parcel update and the
# deposit rules are those of the cuboid mesh, with the wall rule applied per coordinate
# against the box and the owning tet as the cell.

TET_FACES = ((1, 2, 3), (0, 2, 3), (0, 1, 3), (0, 1, 2))


class TetMesh:
    def __init__(self, verts, tets, nbr, L):
        self.v = [tuple(float(a) for a in row) for row in verts]
        self.t, self.nb = [], []
        for k in range(tets.shape[0]):
            order = sorted(range(4), key=lambda j: int(tets[k, j]))
            self.t.append([int(tets[k, j]) for j in order])
            self.nb.append([int(nbr[k, j]) for j in order])
        self.L = float(L)

    def plane(self, t, f):
        v = [self.v[i] for i in self.t[t]]
        p, q, r = (v[j] for j in TET_FACES[f])
        a = [q[k] - p[k] for k in range(3)]
        b = [r[k] - p[k] for k in range(3)]
        n = [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]
        e = (n[0] * (v[f][0] - p[0]) + n[1] * (v[f][1] - p[1])) + n[2] * (v[f][2] - p[2])
        if e > 0.0:
            n = [-n[0], -n[1], -n[2]]
        return n, (n[0] * p[0] + n[1] * p[1]) + n[2] * p[2]

    def walk(self, t, x, hop_limit=64):
        """(tet, hops) or (None, hops) when the walk leaves the mesh or exceeds the limit."""
        hops = 0
        while True:
            s = []
            for f in range(4):
                n, c = self.plane(t, f)
                s.append(((n[0] * x[0] + n[1] * x[1]) + n[2] * x[2]) - c)
            fb = 0
            for f in range(1, 4):
                if s[f] > s[fb]:
                    fb = f
            if not (s[fb] > 0.0):
                return t, hops
            nb = self.nb[t][fb]
            if nb < 0 or hops >= hop_limit:
                return None, hops
            t = nb
            hops += 1


def evolve_parcel_tet(m, prm, pos, vel, cell, dIn, Utet, fs_hi, fs_lo, dtP, dtV, nsteps,
                      mixed, log, hist):
    """One call of the step for one parcel on the tet mesh (positions binary64; velocities
    binary32 in mixed precision, binary64 otherwise)."""
    mu, rho_d, rr, rnu, drag = prm["mu"], prm["rho_d"], prm["rr"], prm["rnu"], prm["drag"]
    if mixed:
        d = F(dIn * F(1.0))
        mB = F(F(F(rr * F(math.pi)) * F(F(d * d) * d)) / F(6))
        f = F(F(F(F(F(18) * mu) * dtV) / F(rho_d * F(d * d))) * F(1.0))
    else:
        d = dIn * 1.0
        mB = ((rr * math.pi) * ((d * d) * d)) / 6.0
        f = ((((18.0 * mu) * dtV) / (rho_d * (d * d)))) * 1.0
    pos, vel = list(pos), list(vel)
    cur = tnew = cell
    Ur = [Utet[cur][c] for c in range(3)]
    state0 = list(vel)
    D = [F(0)] * 3

    def deposit(t, vn):
        if mixed:
            deps = [float(F(mB * D[c])) for c in range(3)]
        else:
            deps = [mB * (state0[c] - vn[c]) for c in range(3)]
        log.append((t + 1, deps))

    for t in range(1, nsteps + 1):
        if mixed:
            sl = [F(fmaf(Ur[c], fs_hi, F(-vel[c])) + F(Ur[c] * fs_lo)) for c in range(3)]
            if drag == 0:
                inc = [F(F(f * sl[c]) / F(F(1) + f)) for c in range(3)]
            else:
                mag = F(np.sqrt(F(F(F(sl[0] * sl[0]) + F(sl[1] * sl[1])) + F(sl[2] * sl[2]))))
                g = F(f * F(F(1) + F(F(0.15) * pow0687f(F(F(mag * d) * rnu)))))
                inc = [F(g * sl[c]) for c in range(3)]
            velNew = [F(vel[c] + inc[c]) for c in range(3)]
        else:
            if drag == 0:
                velNew = [(vel[c] + f * (Ur[c] * fs_hi)) / (1.0 + f) for c in range(3)]
            else:
                du = [Ur[c] * fs_hi - vel[c] for c in range(3)]
                mag = math.sqrt((du[0] * du[0] + du[1] * du[1]) + du[2] * du[2])
                g = f * (1.0 + 0.15 * pow0687((mag * d) * rnu))
                velNew = [vel[c] + g * du[c] for c in range(3)]
        posNew = [pos[c] + float(velNew[c]) * dtP for c in range(3)]
        for c in range(3):
            if posNew[c] < 0.0 or posNew[c] > m.L:
                posNew[c] = pos[c]
                velNew[c] = -vel[c]
                if not mixed:
                    state0[c] = state0[c] - 2.0 * vel[c]
            elif mixed:
                D[c] = F(D[c] - inc[c])
        tnew, hops = m.walk(tnew, posNew)
        assert tnew is not None, "a fixture parcel left the mesh"
        hist[min(hops, 7)] += 1
        if t != nsteps and tnew != cur:
            deposit(cur, velNew)
            state0 = list(velNew)
            D = [F(0)] * 3
            Ur = [Utet[tnew][c] for c in range(3)]
            cur = tnew
        vel, pos = velNew, posNew
    deposit(cur, velNew)
    return pos, vel, tnew


TET_CASES = {
    "tet_sn_sub3_mixed": dict(precision="mixed", seed=41, n=3, npcl=64, drag=1, nsub=3, dt=1e-3,
                              speed=10.0, dmed=40e-6, nsteps=3),
    "tet_stokes_sub2_fp64": dict(precision="fp64", seed=42, n=3, npcl=64, drag=0, nsub=2,
                                 dt=1e-3, speed=20.0, dmed=20e-6, nsteps=3),
}


def run_tet_case(c):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "scale-track_b200"))
    import workload
    mixed = c["precision"] == "mixed"
    vt = np.float32 if mixed else np.float64
    V = F if mixed else float
    L = workload.L_BOX
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(c["n"], L, 0.15, 1)
    rng = np.random.default_rng(c["seed"])
    npcl = c["npcl"]
    xyz = rng.random((3, npcl)) * L
    uvw = rng.normal(0.0, c["speed"], (3, npcl)).astype(vt)
    d = (c["dmed"] * np.exp(0.3 * rng.normal(size=npcl))).astype(vt)
    Utet = (3.0 * (rng.random((tets.shape[0], 3)) * 2.0 - 1.0)).astype(vt)
    hint = workload.tet_hints(xyz, hex_ijk, c["n"], L)
    m = TetMesh(verts, tets, nbr, L)
    cells0 = []
    for i in range(npcl):
        t, _ = m.walk(int(hint[i]), [float(xyz[a, i]) for a in range(3)], hop_limit=1024)
        assert t is not None
        cells0.append(t)
    prm = dict(mu=V(workload.MU_F), rho_d=V(workload.RHO_P), rr=V(workload.RHO_P / workload.RHO_F),
               rnu=V(workload.RHO_F / workload.MU_F), drag=c["drag"])
    Uc = [[V(v) for v in row] for row in Utet]
    fsc = fluid_factors(c["nsteps"])
    dtP = float(c["dt"]) / float(c["nsub"])
    dtV = V(dtP)
    P = [[float(xyz[a, i]) for a in range(3)] for i in range(npcl)]
    W = [[V(uvw[a, i]) for a in range(3)] for i in range(npcl)]
    cells = list(cells0)
    logs, hist = [], [0] * 8
    for s in range(c["nsteps"]):
        fs = float(fsc[s])
        hi = F(fs) if mixed else fs
        lo = F(fs - float(hi)) if mixed else 0.0
        logs.append([])
        for i in range(npcl):
            P[i], W[i], cells[i] = evolve_parcel_tet(m, prm, P[i], W[i], cells[i], V(d[i]), Uc,
                                                     hi, lo, dtP, dtV, c["nsub"], mixed,
                                                     logs[-1], hist)
    nt = tets.shape[0]
    src64 = [[0.0, 0.0, 0.0] for _ in range(nt)]
    for t, comps in logs[-1]:
        for k in range(3):
            src64[t - 1][k] += comps[k]
    return dict(verts=verts, tets=tets, nbr=nbr, xyz0=xyz, uvw0=uvw, d=d, U=Utet, hint=hint,
                cells0=np.array(cells0, dtype=np.int32), fscale=fsc,
                precision=np.array(c["precision"]),
                meta=np.array([c["n"], c["nsub"], c["drag"], c["nsteps"]], dtype=np.int64),
                phys=np.array([L, workload.MU_F, workload.RHO_F, workload.RHO_P, c["dt"]]),
                xyz=np.array(P, dtype=np.float64).T.copy(),
                uvw=np.array(W, dtype=vt).T.copy(),
                cells=np.array(cells, dtype=np.int32),
                hop_hist=np.array(hist, dtype=np.int64),
                src_f64=np.array(src64),
                src_quant=fixed_point_source(logs, nt, npcl, c["nsub"], 1 if mixed else 2))


def main(folder=HERE, verbose=True):
    """Writes every fixture under `folder` (this script's folder by default)."""
    os.makedirs(os.path.join(folder, "tet"), exist_ok=True)
    say = print if verbose else (lambda *a: None)
    for name, c in TET_CASES.items():
        res = run_tet_case(c)
        np.savez(os.path.join(folder, "tet", name + ".npz"), **res)
        say(f"{name}: {c['npcl']} parcels, changed tet {int(np.sum(res['cells'] != res['cells0']))}, "
            f"hops {res['hop_hist'].tolist()}, |src| max {np.abs(res['src_f64']).max():.3e}")
    for name, c in CASES64.items():
        xyz, uvw, d, Ucell = make_inputs64(c["seed"], c["n"], c["npcl"], c["ending"], c["dmin"],
                                           c["dmax"], c["precision"], dlog=c.get("dlog", False))
        fsc = fluid_factors(c["nsteps"])
        res = run_case_p64([c["n"]] * 3, [0.0] * 3, [c["ending"]] * 3, c["mu_c"], c["rho_c"],
                           c["rho_d"], c["drag"], c["nsub"], xyz, uvw, d, Ucell, c["dt"],
                           c["nsteps"], fsc, c["precision"])
        meta = np.array([c["n"], c["nsub"], c["drag"], c["nsteps"]], dtype=np.int64)
        phys = np.array([c["ending"], c["mu_c"], c["rho_c"], c["rho_d"], c["dt"]])
        np.savez(os.path.join(folder, name + ".npz"), meta=meta, phys=phys, xyz0=xyz, uvw0=uvw,
                 d=d, U=Ucell, fscale=fsc, precision=np.array(c["precision"]), **res)
        say(f"{name}: {c['npcl']} parcels, changed cell "
            f"{int(np.sum(res['cells'] != _cells0_64(c, xyz)))}, "
            f"|src| max {np.abs(res['src_f64']).max():.3e}")
    for name, c in CASES.items():
        xyz, uvw, d, Ucell = make_inputs(c["seed"], c["n"], c["npcl"], c["ending"], c["dmin"],
                                         c["dmax"], c.get("v0_random", False))
        res = run_case([c["n"]] * 3, [0.0] * 3, [c["ending"]] * 3, c["mu_c"], c["rho_c"],
                       c["rho_d"], c["drag"], c["nsub"], xyz, uvw, d, Ucell, c["dt"],
                       c["nsteps"])
        meta = np.array([c["n"], c["nsub"], c["drag"], c["nsteps"]], dtype=np.int64)
        phys = np.array([c["ending"], c["mu_c"], c["rho_c"], c["rho_d"], c["dt"]])
        np.savez(os.path.join(folder, name + ".npz"), meta=meta, phys=phys, xyz0=xyz, uvw0=uvw,
                 d=d, U=Ucell, **res)
        say(f"{name}: {c['npcl']} parcels, located {int(np.sum(res['cells'] >= 0))}, "
            f"changed cell {int(np.sum(res['cells'] != _cells0(c, xyz)))}, "
            f"|src| max {np.abs(res['src_f64']).max():.3e}")


if __name__ == "__main__":
    main()
