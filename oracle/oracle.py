"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module; it
is the checker, never the thing measured for the GPU path or shipped in the library.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

PREC = {"fp32": 0, "mixed": 1, "fp64": 2}
DRAG = {"stokes_implicit": 0, "sn_explicit": 1}
INT_MIN = -(2 ** 31)


class OracleCfg(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32 * 3),
        ("origin", ctypes.c_double * 3),
        ("ending", ctypes.c_double * 3),
        ("mu_c", ctypes.c_double),
        ("rho_c", ctypes.c_double),
        ("rho_d", ctypes.c_double),
        ("drag", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("n_substeps", ctypes.c_int32),
        ("quant_limbs", ctypes.c_int32),
        ("drag_multiplier", ctypes.c_double),
        ("diameter_scale", ctypes.c_double),
        ("deposit_bound", ctypes.c_int64),
    ]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.oracle_run.argtypes = [
            P(OracleCfg), ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_double),
            P(ctypes.c_double), P(ctypes.c_double), ctypes.c_int, ctypes.c_double,
            P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_int32),
            P(ctypes.c_int32), P(ctypes.c_int64), ctypes.c_int, P(ctypes.c_int64),
        ]
        L.oracle_run.restype = ctypes.c_int
        L.oracle_locate.argtypes = [P(OracleCfg), ctypes.c_int64, P(ctypes.c_double),
                                    P(ctypes.c_int32)]
        L.oracle_pow0687.argtypes = [ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_double)]
        L.oracle_pow0687f.argtypes = [ctypes.c_int64, P(ctypes.c_float), P(ctypes.c_float)]
        L.oracle_num_threads.restype = ctypes.c_int
        L.oracle_adjoint.argtypes = [
            P(OracleCfg), ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_double),
            P(ctypes.c_double), P(ctypes.c_double), ctypes.c_int, ctypes.c_double,
            P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_int,
            P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double),
            P(ctypes.c_double), P(ctypes.c_int32), P(ctypes.c_uint8), ctypes.c_int]
        L.oracle_adjoint.restype = ctypes.c_int
        L.oracle_tet_run.argtypes = [
            P(OracleCfg), ctypes.c_int64, P(ctypes.c_double), ctypes.c_int64, P(ctypes.c_int32),
            P(ctypes.c_int32), ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_double),
            P(ctypes.c_double), P(ctypes.c_int32), P(ctypes.c_double), ctypes.c_int,
            ctypes.c_double, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_double),
            P(ctypes.c_int32), P(ctypes.c_int64), P(ctypes.c_int64), ctypes.c_int]
        L.oracle_tet_run.restype = ctypes.c_int
        L.oracle_tet_locate.argtypes = [
            ctypes.c_int64, P(ctypes.c_double), ctypes.c_int64, P(ctypes.c_int32),
            P(ctypes.c_int32), ctypes.c_int64, P(ctypes.c_double), P(ctypes.c_int32),
            P(ctypes.c_int32), P(ctypes.c_int32), ctypes.c_int]
        L.oracle_init_parcels.argtypes = [
            ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
            P(ctypes.c_int32), P(ctypes.c_double), P(ctypes.c_double), ctypes.c_double,
            ctypes.c_double, P(ctypes.c_double), P(ctypes.c_double)]
        L.oracle_hilbert3.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def make_cfg(n, origin, ending, mu_c, rho_c, rho_d, drag="sn_explicit", precision="mixed",
             n_substeps=1, quant_limbs=1, drag_multiplier=1.0, diameter_scale=1.0,
             deposit_bound=0):
    c = OracleCfg()
    n = [n] * 3 if np.isscalar(n) else list(n)
    origin = [origin] * 3 if np.isscalar(origin) else list(origin)
    ending = [ending] * 3 if np.isscalar(ending) else list(ending)
    c.n = (ctypes.c_int32 * 3)(*n)
    c.origin = (ctypes.c_double * 3)(*origin)
    c.ending = (ctypes.c_double * 3)(*ending)
    c.mu_c, c.rho_c, c.rho_d = mu_c, rho_c, rho_d
    c.drag = DRAG[drag] if isinstance(drag, str) else int(drag)
    c.precision = PREC[precision] if isinstance(precision, str) else int(precision)
    c.n_substeps = n_substeps
    c.quant_limbs = quant_limbs
    c.drag_multiplier = drag_multiplier
    c.diameter_scale = diameter_scale
    c.deposit_bound = deposit_bound
    return c


def run(cfg, xyz, uvw, d, U, nsteps, dt, fscale=None, want_seq=True, want_quant=True,
        scale=INT_MIN, nthreads=1, want_acc=False):
    """Runs nsteps steps.  xyz/uvw are [3, np] float64 (copied), d [np], U [ncells, 3].
    nsteps=0 with scale=INT_MIN runs the first step's probe only (its exponent in "emax").

    Returns dict(xyz, uvw, cells, src_seq, src_quant, scale, lost, overflow, H, emax, acc,
    status); emax is the largest-deposit exponent of the last step, acc (want_acc) its raw
    int64 fixed-point accumulators."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
    uvw = np.ascontiguousarray(uvw, dtype=np.float64).copy()
    d = np.ascontiguousarray(d, dtype=np.float64)
    U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
    npcl = d.shape[0]
    ncells = int(cfg.n[0]) * int(cfg.n[1]) * int(cfg.n[2])
    assert U.shape[0] == 3 * ncells
    fs = None if fscale is None else np.ascontiguousarray(fscale, dtype=np.float64)
    src_seq = np.zeros(3 * ncells) if want_seq else None
    src_q = np.zeros(3 * ncells) if want_quant else None
    cells = np.zeros(npcl, dtype=np.int32)
    sc = np.array([scale], dtype=np.int32)
    stats = np.zeros(4, dtype=np.int64)
    acc = np.zeros(3 * ncells * cfg.quant_limbs, dtype=np.int64) if want_acc else None
    st = lib().oracle_run(ctypes.byref(cfg), npcl, _ptr(xyz, ctypes.c_double),
                          _ptr(uvw, ctypes.c_double), _ptr(d, ctypes.c_double),
                          _ptr(U, ctypes.c_double), nsteps, dt, _ptr(fs, ctypes.c_double),
                          _ptr(src_seq, ctypes.c_double), _ptr(src_q, ctypes.c_double),
                          _ptr(cells, ctypes.c_int32), _ptr(sc, ctypes.c_int32),
                          _ptr(stats, ctypes.c_int64), nthreads, _ptr(acc, ctypes.c_int64))
    return dict(xyz=xyz, uvw=uvw, cells=cells,
                src_seq=None if src_seq is None else src_seq.reshape(ncells, 3),
                src_quant=None if src_q is None else src_q.reshape(ncells, 3),
                scale=int(sc[0]), lost=int(stats[0]), overflow=int(stats[1]), H=int(stats[2]),
                emax=int(stats[3]), acc=acc, status=st)


def locate(cfg, xyz):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    npcl = xyz.shape[1]
    cells = np.zeros(npcl, dtype=np.int32)
    lib().oracle_locate(ctypes.byref(cfg), npcl, _ptr(xyz, ctypes.c_double),
                        _ptr(cells, ctypes.c_int32))
    return cells


def pow0687(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    lib().oracle_pow0687(x.size, _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double))
    return y


def pow0687f(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.empty_like(x)
    lib().oracle_pow0687f(x.size, _ptr(x, ctypes.c_float), _ptr(y, ctypes.c_float))
    return y


def num_threads():
    return lib().oracle_num_threads()


def adjoint(cfg, xyz, uvw, d, U, T, dt, fscale=None, cotangent=None, target=None,
            mean_limbs=1, grad=True, frozen=None):
    """Mean-source objective (and its adjoint when grad=True) with frozen ownership.

    frozen=None records the ownership of this run; frozen=(cells, bounce) replays it.
    Returns dict(mean_src, J, dalpha, dscale, dv0 [3, np], frozen=(cells, bounce), status)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    uvw = np.ascontiguousarray(uvw, dtype=np.float64)
    d = np.ascontiguousarray(d, dtype=np.float64)
    U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
    npcl = d.shape[0]
    ncells = int(cfg.n[0]) * int(cfg.n[1]) * int(cfg.n[2])
    fs = None if fscale is None else np.ascontiguousarray(fscale, dtype=np.float64)
    cot = None if cotangent is None else np.ascontiguousarray(cotangent, dtype=np.float64).reshape(-1)
    tgt = None if target is None else np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
    mean = np.zeros(3 * ncells)
    J = np.zeros(1)
    da = np.zeros(1)
    ds = np.zeros(1)
    dv0 = np.zeros((3, npcl)) if grad else None
    replay = frozen is not None
    if replay:
        cells = np.ascontiguousarray(frozen[0], dtype=np.int32)
        bounce = np.ascontiguousarray(frozen[1], dtype=np.uint8)
    else:
        cells = np.zeros(T * npcl, dtype=np.int32)
        bounce = np.zeros(T * npcl, dtype=np.uint8)
    st = lib().oracle_adjoint(ctypes.byref(cfg), npcl, _ptr(xyz, ctypes.c_double),
                              _ptr(uvw, ctypes.c_double), _ptr(d, ctypes.c_double),
                              _ptr(U, ctypes.c_double), T, dt, _ptr(fs, ctypes.c_double),
                              _ptr(cot, ctypes.c_double), _ptr(tgt, ctypes.c_double), mean_limbs,
                              _ptr(mean, ctypes.c_double), _ptr(J, ctypes.c_double),
                              _ptr(da, ctypes.c_double) if grad else None,
                              _ptr(ds, ctypes.c_double) if grad else None,
                              _ptr(dv0, ctypes.c_double), _ptr(cells, ctypes.c_int32),
                              _ptr(bounce, ctypes.c_uint8), 1 if replay else 0)
    return dict(mean_src=mean.reshape(ncells, 3), J=float(J[0]), dalpha=float(da[0]),
                dscale=float(ds[0]), dv0=dv0, frozen=(cells, bounce), status=st)


def tet_run(cfg, mesh, xyz, uvw, d, cells, U, nsteps, dt, fscale=None, want_seq=True,
            want_quant=True, scale=INT_MIN, hop_limit=64):
    """Steps on a tet mesh (verts, tets, nbrs); cells [np] start tets.  Returns dict(xyz, uvw,
    cells, src_seq, src_quant, scale, lost, overflow, hop_hist, status)."""
    verts, tets, nbrs = (np.ascontiguousarray(mesh[0], dtype=np.float64),
                         np.ascontiguousarray(mesh[1], dtype=np.int32),
                         np.ascontiguousarray(mesh[2], dtype=np.int32))
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).copy()
    uvw = np.ascontiguousarray(uvw, dtype=np.float64).copy()
    d = np.ascontiguousarray(d, dtype=np.float64)
    cells = np.ascontiguousarray(cells, dtype=np.int32).copy()
    U = np.ascontiguousarray(U, dtype=np.float64).reshape(-1)
    nt = tets.shape[0]
    fs = None if fscale is None else np.ascontiguousarray(fscale, dtype=np.float64)
    src_seq = np.zeros(3 * nt) if want_seq else None
    src_q = np.zeros(3 * nt) if want_quant else None
    sc = np.array([scale], dtype=np.int32)
    stats = np.zeros(3, dtype=np.int64)
    hist = np.zeros(8, dtype=np.int64)
    st = lib().oracle_tet_run(ctypes.byref(cfg), verts.shape[0], _ptr(verts, ctypes.c_double),
                              nt, _ptr(tets, ctypes.c_int32), _ptr(nbrs, ctypes.c_int32),
                              d.shape[0], _ptr(xyz, ctypes.c_double), _ptr(uvw, ctypes.c_double),
                              _ptr(d, ctypes.c_double), _ptr(cells, ctypes.c_int32),
                              _ptr(U, ctypes.c_double), nsteps, dt, _ptr(fs, ctypes.c_double),
                              _ptr(src_seq, ctypes.c_double), _ptr(src_q, ctypes.c_double),
                              _ptr(sc, ctypes.c_int32), _ptr(stats, ctypes.c_int64),
                              _ptr(hist, ctypes.c_int64), hop_limit)
    return dict(xyz=xyz, uvw=uvw, cells=cells,
                src_seq=None if src_seq is None else src_seq.reshape(nt, 3),
                src_quant=None if src_q is None else src_q.reshape(nt, 3), scale=int(sc[0]),
                lost=int(stats[0]), overflow=int(stats[1]), hop_hist=hist, status=st)


def init_parcels(pbytes, seed, cloud, nclouds, n, N, origin, ending, d_min, d_max):
    """Parcels of st_init_parcels: (xyz [3, n] rounded to the position precision, d [n])."""
    N = (ctypes.c_int32 * 3)(*([N] * 3 if np.isscalar(N) else list(N)))
    o = (ctypes.c_double * 3)(*([origin] * 3 if np.isscalar(origin) else list(origin)))
    e = (ctypes.c_double * 3)(*([ending] * 3 if np.isscalar(ending) else list(ending)))
    xyz = np.zeros((3, n))
    d = np.zeros(n)
    lib().oracle_init_parcels(pbytes, ctypes.c_uint64(seed), cloud, nclouds, n, N, o, e,
                              ctypes.c_double(d_min), ctypes.c_double(d_max),
                              _ptr(xyz, ctypes.c_double), _ptr(d, ctypes.c_double))
    return xyz, d


def hilbert3(h, bits):
    h = np.ascontiguousarray(h, dtype=np.uint64)
    p = np.zeros((h.size, 3), dtype=np.uint32)
    lib().oracle_hilbert3(h.size, h.ctypes.data_as(ctypes.c_void_p), bits,
                          p.ctypes.data_as(ctypes.c_void_p))
    return p


def tet_locate(mesh, xyz, start, hop_limit=1024):
    verts, tets, nbrs = (np.ascontiguousarray(mesh[0], dtype=np.float64),
                         np.ascontiguousarray(mesh[1], dtype=np.int32),
                         np.ascontiguousarray(mesh[2], dtype=np.int32))
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    start = np.ascontiguousarray(start, dtype=np.int32)
    npcl = xyz.shape[1]
    cells = np.zeros(npcl, dtype=np.int32)
    status = np.zeros(npcl, dtype=np.int32)
    lib().oracle_tet_locate(verts.shape[0], _ptr(verts, ctypes.c_double), tets.shape[0],
                            _ptr(tets, ctypes.c_int32), _ptr(nbrs, ctypes.c_int32), npcl,
                            _ptr(xyz, ctypes.c_double), _ptr(start, ctypes.c_int32),
                            _ptr(cells, ctypes.c_int32), _ptr(status, ctypes.c_int32),
                            hop_limit)
    return cells, status
