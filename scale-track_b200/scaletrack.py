"""Python host side of libscaletrack.so (ctypes), mirroring the reference's coupling surface.

The reference's host language for this path is Julia calling CUDA.jl kernels, driven by an
OpenFOAM solver through two C function pointers (allocate_array_ptr and evolve_cloud_ptr,
A:1436-1528).  Julia is not available here, so this module is the host used by the tests
and the benchmark; it calls the same C ABI that a Julia `ccall` or the C++ solver would
(see include/scaletrack.h).  There is no CPU fallback: if the shared library or a CUDA
device is missing, the calls raise.

    A: run/icoJuliaParcelFoam/cavity3D/asyncParallelTracking.jl
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SCALETRACK_LIB") or os.path.join(HERE, "libscaletrack.so")

ST_OK = 0
ST_ERR_INVALID_ARGUMENT = 1
ST_ERR_CUDA = 2
ST_ERR_PARCEL_OUTSIDE = 3
ST_ERR_SOURCE_RANGE = 4
ST_ERR_NOT_INITIALISED = 5
ST_ERR_OUT_OF_MEMORY = 6

DRAG = {"stokes_implicit": 0, "schiller_naumann": 1, "sn_explicit": 1}
PRECISION = {"fp32": 0, "mixed": 1, "fp64": 2}
DEPOSIT = {"deterministic": 0, "atomic": 1}
KERNEL_KINDS = {"step": 0, "finalize": 1, "sort": 2, "probe": 3, "other": 4,
                "adj_forward": 5, "adj_reverse": 6}

# every symbol include/scaletrack.h declares
EXPORTS = [
    "st_version", "st_last_error", "st_params_default", "st_create", "st_destroy",
    "st_set_parcels", "st_get_parcels", "st_get_cells", "st_get_order", "st_num_parcels",
    "st_get_parcel_sample",
    "st_num_cells",
    "st_set_fluid_velocity", "st_set_fluid_velocity_device", "st_step", "st_get_source",
    "st_source_device", "st_synchronize", "st_get_stream", "st_set_stream",
    "st_profile_enable", "st_profile_read", "st_launch_count", "st_set_step_kernel", "st_set_finalize_overlap", "st_set_wait_limit",
    "st_setup",
    "st_set_drag_parameters", "st_shard_set_total", "st_shard_buffers", "st_shard_needs_probe",
    "st_shard_probe", "st_shard_deposit", "st_shard_finish",
    "st_default_handle",
    "st_allocate_array", "st_evolve_cloud", "st_finalize", "st_step_noalloc",
    "st_noalloc_max_cells", "st_mean_source_forward", "st_mean_source_pullback",
    "st_graph_capture", "st_graph_launch", "st_graph_release", "st_autotune",
    "st_create_tet", "st_set_parcels_tet", "st_tet_hop_histogram", "st_evolve_cloud_async",
    "st_init_parcels", "st_write_vtu", "st_write_pvd", "st_save_state", "st_load_state",
    "st_set_exchange_mode", "st_append_parcels",
]


class ScaleTrackError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"scaletrack error {code}: {msg}")
        self.code = code


class MeshDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32 * 3), ("origin", ctypes.c_double * 3),
                ("ending", ctypes.c_double * 3)]


class TetMeshDesc(ctypes.Structure):
    _fields_ = [("n_vertices", ctypes.c_int64), ("vertices", ctypes.c_void_p),
                ("n_tets", ctypes.c_int64), ("tets", ctypes.c_void_p),
                ("neighbors", ctypes.c_void_p), ("origin", ctypes.c_double * 3),
                ("ending", ctypes.c_double * 3), ("hop_limit", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


class Params(ctypes.Structure):
    _fields_ = [
        ("mu_c", ctypes.c_double), ("rho_c", ctypes.c_double), ("rho_d", ctypes.c_double),
        ("drag_model", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("deposit", ctypes.c_int32), ("n_substeps", ctypes.c_int32),
        ("sort_interval", ctypes.c_int32), ("n_clouds", ctypes.c_int32),
        ("block_size", ctypes.c_int32), ("grid_blocks", ctypes.c_int32),
        ("drag_multiplier", ctypes.c_double), ("diameter_scale", ctypes.c_double),
    ]


class TuneResult(ctypes.Structure):
    _fields_ = [("block_size", ctypes.c_int32), ("grid_blocks", ctypes.c_int32),
                ("sort_interval", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("ms_per_step", ctypes.c_double)]


class AdjointDesc(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int32), ("checkpoint_interval", ctypes.c_int32),
                ("dt", ctypes.c_double), ("fluid_scale", ctypes.POINTER(ctypes.c_double))]


_lib = None


def lib():
    """Loads libscaletrack.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ScaleTrackError(-1, f"{LIB_PATH} is missing: run scale-track_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    c_h = ctypes.c_void_p
    sig = {
        "st_version": ([], ctypes.c_char_p),
        "st_last_error": ([], ctypes.c_char_p),
        "st_params_default": ([P(Params)], None),
        "st_create": ([P(Params), P(MeshDesc), ctypes.c_int, P(c_h)], ctypes.c_int),
        "st_destroy": ([c_h], ctypes.c_int),
        "st_set_parcels": ([c_h, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
        "st_get_parcels": ([c_h, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p], ctypes.c_int),
        "st_get_cells": ([c_h, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
        "st_get_order": ([c_h, ctypes.c_int, ctypes.c_void_p], ctypes.c_int),
        "st_get_parcel_sample": ([c_h, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                                 ctypes.c_int),
        "st_num_parcels": ([c_h, ctypes.c_int], ctypes.c_int64),
        "st_num_cells": ([c_h], ctypes.c_int64),
        "st_set_fluid_velocity": ([c_h, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "st_set_fluid_velocity_device": ([c_h, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "st_step": ([c_h, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "st_get_source": ([c_h, ctypes.c_int, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "st_source_device": ([c_h, ctypes.c_int], ctypes.c_void_p),
        "st_synchronize": ([c_h], ctypes.c_int),
        "st_get_stream": ([c_h], ctypes.c_void_p),
        "st_set_stream": ([c_h, ctypes.c_void_p], ctypes.c_int),
        "st_profile_enable": ([c_h, ctypes.c_int], ctypes.c_int),
        "st_profile_read": ([c_h, ctypes.c_int, P(ctypes.c_int64), P(ctypes.c_double),
                             ctypes.c_int], ctypes.c_int),
        "st_launch_count": ([c_h], ctypes.c_int64),
        "st_set_step_kernel": ([c_h, ctypes.c_int], ctypes.c_int),
        "st_set_finalize_overlap": ([c_h, ctypes.c_int], ctypes.c_int),
        "st_set_wait_limit": ([c_h, ctypes.c_int64, ctypes.c_int], ctypes.c_int),
        "st_set_drag_parameters": ([c_h, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "st_shard_set_total": ([c_h, ctypes.c_int, ctypes.c_int64], ctypes.c_int),
        "st_shard_buffers": ([c_h, P(ctypes.c_void_p), P(ctypes.c_int64), P(ctypes.c_void_p),
                              P(ctypes.c_int32)], ctypes.c_int),
        "st_shard_needs_probe": ([c_h, ctypes.c_double], ctypes.c_int),
        "st_shard_probe": ([c_h, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "st_shard_deposit": ([c_h, ctypes.c_double, ctypes.c_double], ctypes.c_int),
        "st_shard_finish": ([c_h], ctypes.c_int),
        "st_setup": ([P(Params), P(MeshDesc)], ctypes.c_int),
        "st_default_handle": ([], c_h),
        "st_allocate_array": ([ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int],
                              ctypes.c_void_p),
        "st_evolve_cloud": ([ctypes.c_double], ctypes.c_int),
        "st_evolve_cloud_async": ([ctypes.c_double], ctypes.c_int),
        "st_set_exchange_mode": ([ctypes.c_int], ctypes.c_int),
        "st_append_parcels": ([c_h, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
        "st_write_vtu": ([c_h, ctypes.c_int, ctypes.c_char_p], ctypes.c_int),
        "st_write_pvd": ([ctypes.c_char_p, ctypes.c_int, P(ctypes.c_double),
                          P(ctypes.c_char_p)], ctypes.c_int),
        "st_save_state": ([c_h, ctypes.c_char_p], ctypes.c_int),
        "st_load_state": ([c_h, ctypes.c_char_p], ctypes.c_int),
        "st_init_parcels": ([c_h, ctypes.c_int, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double,
                             ctypes.c_double], ctypes.c_int),
        "st_finalize": ([], ctypes.c_int),
        "st_step_noalloc": ([P(Params), P(MeshDesc), ctypes.c_int64] + [ctypes.c_void_p] * 9 +
                            [ctypes.c_double, ctypes.c_double, ctypes.c_void_p], ctypes.c_int),
        "st_noalloc_max_cells": ([], ctypes.c_int64),
        "st_graph_capture": ([c_h, ctypes.c_int, ctypes.c_double, ctypes.c_void_p],
                             ctypes.c_int),
        "st_graph_launch": ([c_h], ctypes.c_int),
        "st_graph_release": ([c_h], ctypes.c_int),
        "st_autotune": ([c_h, ctypes.c_double, ctypes.c_int, P(TuneResult)], ctypes.c_int),
        "st_create_tet": ([P(Params), P(TetMeshDesc), ctypes.c_int, P(c_h)], ctypes.c_int),
        "st_set_parcels_tet": ([c_h, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                               ctypes.c_int),
        "st_tet_hop_histogram": ([c_h, ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
        "st_mean_source_forward": ([c_h, ctypes.c_int, P(AdjointDesc), ctypes.c_void_p],
                                   ctypes.c_int),
        "st_mean_source_pullback": ([c_h, ctypes.c_int, P(AdjointDesc), ctypes.c_void_p,
                                     P(ctypes.c_double), P(ctypes.c_double), ctypes.c_void_p],
                                    ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def last_error():
    return lib().st_last_error().decode()


def _check(rc):
    if rc != ST_OK:
        raise ScaleTrackError(rc, last_error())
    return rc


def _vec3(v):
    return [v] * 3 if np.isscalar(v) else list(v)


def mesh_desc(n, origin, ending):
    """Uniform cuboid mesh; like the reference's Mesh(N, origin, ending) (A:259-268)."""
    m = MeshDesc()
    m.n = (ctypes.c_int32 * 3)(*[int(x) for x in _vec3(n)])
    m.origin = (ctypes.c_double * 3)(*[float(x) for x in _vec3(origin)])
    m.ending = (ctypes.c_double * 3)(*[float(x) for x in _vec3(ending)])
    return m


def tet_mesh_desc(vertices, tets, neighbors, origin, ending, hop_limit=0):
    """Tetrahedral mesh filling the box [origin, ending]: vertices [nv][3] (FP64), tets and
    neighbours [nt][4] (int32; neighbour across the face opposite local vertex f, -1 on
    the boundary).  The returned descriptor keeps the arrays alive."""
    verts = np.ascontiguousarray(vertices, dtype=np.float64)
    tt = np.ascontiguousarray(tets, dtype=np.int32)
    nb = np.ascontiguousarray(neighbors, dtype=np.int32)
    if verts.ndim != 2 or verts.shape[1] != 3:
        raise ValueError("vertices must be [nv][3]")
    if tt.shape != nb.shape or tt.ndim != 2 or tt.shape[1] != 4:
        raise ValueError("tets and neighbors must both be [nt][4]")
    m = TetMeshDesc()
    m.n_vertices = verts.shape[0]
    m.vertices = verts.ctypes.data
    m.n_tets = tt.shape[0]
    m.tets = tt.ctypes.data
    m.neighbors = nb.ctypes.data
    m.origin = (ctypes.c_double * 3)(*[float(x) for x in _vec3(origin)])
    m.ending = (ctypes.c_double * 3)(*[float(x) for x in _vec3(ending)])
    m.hop_limit = int(hop_limit)
    m._keep = (verts, tt, nb)
    return m


def params(**kw):
    """st_params with the library defaults (the reference's setup.jl) overridden by kw.
    String values are accepted for drag_model, precision and deposit."""
    p = Params()
    lib().st_params_default(ctypes.byref(p))
    for k, v in kw.items():
        if k == "drag_model" and isinstance(v, str):
            v = DRAG[v]
        elif k == "precision" and isinstance(v, str):
            v = PRECISION[v]
        elif k == "deposit" and isinstance(v, str):
            v = DEPOSIT[v]
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


def _check_parcel_shapes(xyz, uvw, n):
    if xyz.shape != (3, n) or uvw.shape != (3, n):
        raise ValueError(f"xyz and uvw must be [3][{n}] (one column per parcel), got "
                         f"{xyz.shape} and {uvw.shape}")


def _dptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class ParcelTracker:
    """One handle: a mesh, its cell fields and n_clouds parcel clouds on one GPU."""

    def __init__(self, prm, mesh, device=0):
        self._h = ctypes.c_void_p()
        self.params = prm
        self.mesh = mesh
        self.tet = isinstance(mesh, TetMeshDesc)
        create = lib().st_create_tet if self.tet else lib().st_create
        _check(create(ctypes.byref(prm), ctypes.byref(mesh), device, ctypes.byref(self._h)))
        self.ncells = int(lib().st_num_cells(self._h))

    def close(self):
        if self._h:
            lib().st_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_parcels(self, xyz, uvw, d, cloud=0, hint=None):
        """hint: starting tet per parcel for the walk to the owning tet (tet meshes only)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        uvw = np.ascontiguousarray(uvw, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        n = d.shape[0]
        _check_parcel_shapes(xyz, uvw, n)
        if self.tet:
            h = None if hint is None else np.ascontiguousarray(hint, dtype=np.int32)
            if h is not None and h.shape != (n,):
                raise ValueError("hint must hold one starting tet per parcel")
            _check(lib().st_set_parcels_tet(self._h, cloud, n, _dptr(xyz), _dptr(uvw),
                                            _dptr(d), _dptr(h)))
        else:
            if hint is not None:
                raise ValueError("hint is for tet meshes")
            _check(lib().st_set_parcels(self._h, cloud, n, _dptr(xyz), _dptr(uvw), _dptr(d)))

    def hop_histogram(self, reset=False):
        """Walk lengths per substep since the last reset: [k] = walks of k hops, [7] = 7+."""
        out = np.zeros(8, dtype=np.uint64)
        _check(lib().st_tet_hop_histogram(self._h, _dptr(out), int(reset)))
        return out

    def append_parcels(self, xyz, uvw, d, cloud=0):
        """Injection: parcels added to the end of a cloud, in place on the device."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        uvw = np.ascontiguousarray(uvw, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.float64)
        m = d.shape[0]
        _check_parcel_shapes(xyz, uvw, m)
        _check(lib().st_append_parcels(self._h, cloud, m, _dptr(xyz), _dptr(uvw), _dptr(d)))

    def init_parcels(self, n, seed, d_min, d_max, cloud=0):
        """n parcels generated on the device, clustered along a Hilbert curve per cloud."""
        _check(lib().st_init_parcels(self._h, cloud, n, seed, d_min, d_max))

    def write_vtu(self, path, cloud=0):
        """ParaView dump of a cloud: positions, point data U (velocity) and d (diameter)."""
        _check(lib().st_write_vtu(self._h, cloud, os.fsencode(path)))

    def save_state(self, path):
        _check(lib().st_save_state(self._h, os.fsencode(path)))

    def load_state(self, path):
        _check(lib().st_load_state(self._h, os.fsencode(path)))

    def num_parcels(self, cloud=0):
        n = int(lib().st_num_parcels(self._h, cloud))
        if n < 0:
            raise ScaleTrackError(ST_ERR_INVALID_ARGUMENT, f"cloud {cloud} out of range")
        return n

    def get_parcels(self, cloud=0, check=True):
        n = self.num_parcels(cloud)
        xyz = np.empty((3, n))
        uvw = np.empty((3, n))
        d = np.empty(n)
        rc = lib().st_get_parcels(self._h, cloud, _dptr(xyz), _dptr(uvw), _dptr(d))
        if check:
            _check(rc)
        return xyz, uvw, d

    def get_cells(self, cloud=0, check=True):
        n = self.num_parcels(cloud)
        cells = np.empty(n, dtype=np.int32)
        rc = lib().st_get_cells(self._h, cloud, _dptr(cells))
        if check:
            _check(rc)
        return cells

    def get_parcel_sample(self, ids, cloud=0):
        """(xyz [3, m], uvw [3, m], cells [m]) of the parcels with st_set_parcels indices ids"""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        m = ids.shape[0]
        xyz = np.empty((3, m))
        uvw = np.empty((3, m))
        cells = np.empty(m, dtype=np.int32)
        _check(lib().st_get_parcel_sample(self._h, cloud, m, _dptr(ids), _dptr(xyz), _dptr(uvw),
                                          _dptr(cells)))
        return xyz, uvw, cells

    def get_order(self, cloud=0):
        """ids[k]: st_set_parcels index of the parcel at device position k."""
        ids = np.empty(self.num_parcels(cloud), dtype=np.int32)
        _check(lib().st_get_order(self._h, cloud, _dptr(ids)))
        return ids

    def set_fluid_velocity(self, U):
        U = np.ascontiguousarray(U)
        if U.shape != (self.ncells, 3) or U.dtype not in (np.float32, np.float64):
            raise ValueError(f"U must be float32 or float64 [{self.ncells}][3], got "
                             f"{U.dtype} {U.shape}")
        _check(lib().st_set_fluid_velocity(self._h, _dptr(U), U.dtype.itemsize))

    def set_fluid_velocity_device(self, ptr, elem_bytes):
        _check(lib().st_set_fluid_velocity_device(self._h, ctypes.c_void_p(ptr), elem_bytes))

    def step(self, dt, fluid_scale=1.0):
        _check(lib().st_step(self._h, dt, fluid_scale))

    def get_source(self, cloud=0, dtype=np.float64, check=True):
        S = np.empty((self.ncells, 3), dtype=dtype)
        rc = lib().st_get_source(self._h, cloud, _dptr(S), S.dtype.itemsize)
        if check:
            _check(rc)
        return S

    def source_device_ptr(self, cloud=0):
        return lib().st_source_device(self._h, cloud)

    def synchronize(self):
        _check(lib().st_synchronize(self._h))

    def stream(self):
        """The handle's cudaStream_t as an int (0: the legacy default stream, e.g. after
        st_set_stream with torch's default stream)."""
        return lib().st_get_stream(self._h) or 0

    def profile(self, on=True):
        _check(lib().st_profile_enable(self._h, 1 if on else 0))

    def profile_read(self, kind, reset=False):
        n = ctypes.c_int64()
        ms = ctypes.c_double()
        k = KERNEL_KINDS[kind] if isinstance(kind, str) else kind
        _check(lib().st_profile_read(self._h, k, ctypes.byref(n), ctypes.byref(ms),
                                     1 if reset else 0))
        return int(n.value), float(ms.value)

    def launch_count(self):
        return int(lib().st_launch_count(self._h))

    # ---- sharded steps (one cloud split over ranks) -------------------------------
    def shard_set_total(self, n_parcels_all_ranks, cloud=0):
        _check(lib().st_shard_set_total(self._h, cloud, int(n_parcels_all_ranks)))

    def shard_buffers(self):
        """(accumulator device pointer, int64 count, exponent device pointer, int32 count)"""
        acc, nacc = ctypes.c_void_p(), ctypes.c_int64()
        ex, nex = ctypes.c_void_p(), ctypes.c_int32()
        _check(lib().st_shard_buffers(self._h, ctypes.byref(acc), ctypes.byref(nacc),
                                      ctypes.byref(ex), ctypes.byref(nex)))
        return acc.value, nacc.value, ex.value, nex.value

    def shard_needs_probe(self, dt):
        r = lib().st_shard_needs_probe(self._h, dt)
        if r < 0:
            _check(r)
        return bool(r)

    def shard_probe(self, dt, fluid_scale=1.0):
        _check(lib().st_shard_probe(self._h, dt, fluid_scale))

    def shard_deposit(self, dt, fluid_scale=1.0):
        _check(lib().st_shard_deposit(self._h, dt, fluid_scale))

    def shard_finish(self):
        _check(lib().st_shard_finish(self._h))

    def set_drag_parameters(self, drag_multiplier, diameter_scale):
        _check(lib().st_set_drag_parameters(self._h, drag_multiplier, diameter_scale))

    def set_finalize_overlap(self, on):
        """Overlap each step's source conversion with the next step (default on)."""
        _check(lib().st_set_finalize_overlap(self._h, 1 if on else 0))

    def set_wait_limit(self, cycles, stall=False):
        """Limit of the ring kernels' pipeline waits in SM clock cycles (0 = about 1 s);
        stall=True makes the waits run out (failure-detection test)."""
        _check(lib().st_set_wait_limit(self._h, int(cycles), 1 if stall else 0))

    def set_step_kernel(self, kind):
        """'ring' (default: shared-memory ring of block tiles) or 'warp' (per-warp tiles);
        both give bit-identical results."""
        k = {"ring": 0, "warp": 1}[kind] if isinstance(kind, str) else int(kind)
        _check(lib().st_set_step_kernel(self._h, k))

    def graph_capture(self, n_steps, dt, fluid_scale=None):
        fs = None if fluid_scale is None else np.ascontiguousarray(fluid_scale, dtype=np.float64)
        _check(lib().st_graph_capture(self._h, n_steps, dt, _dptr(fs)))

    def graph_launch(self):
        _check(lib().st_graph_launch(self._h))

    def graph_release(self):
        _check(lib().st_graph_release(self._h))

    def autotune(self, dt, trial_steps=40):
        r = TuneResult()
        _check(lib().st_autotune(self._h, dt, trial_steps, ctypes.byref(r)))
        return dict(block_size=r.block_size, grid_blocks=r.grid_blocks,
                    sort_interval=r.sort_interval, ms_per_step=r.ms_per_step)

    def _adj_desc(self, n_steps, checkpoint_interval, dt, fluid_scale):
        fs = None
        if fluid_scale is not None:
            fs = np.ascontiguousarray(fluid_scale, dtype=np.float64)
            if fs.shape != (n_steps,):
                raise ValueError("fluid_scale must hold one factor per step")
        desc = AdjointDesc(n_steps, checkpoint_interval, dt,
                           None if fs is None else fs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return desc, fs

    def mean_source_forward(self, n_steps, checkpoint_interval, dt, fluid_scale=None, cloud=0):
        """Sbar = (1/T) sum of the per-step sources over T steps from the current state (the
        state is not modified); keeps the checkpoints for mean_source_pullback."""
        desc, keep = self._adj_desc(n_steps, checkpoint_interval, dt, fluid_scale)
        S = np.empty((self.ncells, 3))
        _check(lib().st_mean_source_forward(self._h, cloud, ctypes.byref(desc), _dptr(S)))
        return S

    def mean_source_pullback(self, cotangent, n_steps, checkpoint_interval, dt,
                             fluid_scale=None, cloud=0, want_v0=True):
        """Pull-back of the last mean_source_forward: (dJ/dalpha, dJ/ds, dJ/dv0 [3, n])."""
        desc, keep = self._adj_desc(n_steps, checkpoint_interval, dt, fluid_scale)
        cot = np.ascontiguousarray(cotangent, dtype=np.float64).reshape(self.ncells, 3)
        da = ctypes.c_double()
        ds = ctypes.c_double()
        dv0 = np.empty((3, self.num_parcels(cloud))) if want_v0 else None
        _check(lib().st_mean_source_pullback(self._h, cloud, ctypes.byref(desc), _dptr(cot),
                                             ctypes.byref(da), ctypes.byref(ds), _dptr(dv0)))
        return float(da.value), float(ds.value), dv0


# ---------------------------------------------------------------------------------------
# the reference's coupling surface (process-wide default handle)
# ---------------------------------------------------------------------------------------
def setup(prm, mesh):
    """Creates the default handle used by allocate_array and evolve_cloud."""
    _check(lib().st_setup(ctypes.byref(prm), ctypes.byref(mesh)))


def default_handle():
    return lib().st_default_handle()


def allocate_array(name, size, n_components, type_byte_size):
    """allocate_array_ptr (A:1436-1483): library-owned pinned storage [size][n_components]
    returned as a numpy view, which the caller fills (U) or reads (UTrans) in place."""
    p = lib().st_allocate_array(name.encode(), size, n_components, type_byte_size)
    if not p:
        raise ScaleTrackError(ST_ERR_INVALID_ARGUMENT, last_error())
    ctype = ctypes.c_float if type_byte_size == 4 else ctypes.c_double
    buf = (ctype * (size * n_components)).from_address(p)
    return np.ctypeslib.as_array(buf).reshape(size, n_components)


def evolve_cloud(dt):
    """evolve_cloud (A:1485-1528): one synchronous step on the default handle."""
    _check(lib().st_evolve_cloud(dt))


def evolve_cloud_async(dt):
    """The reference's asynchronous coupling: U is taken, UTrans receives the constant
    extrapolation 2 S_prev - est_prev of the source, and this step runs in the background."""
    _check(lib().st_evolve_cloud_async(dt))


def write_pvd(path, times, files):
    """ParaView collection of dumps: times[i] -> files[i]."""
    n = len(times)
    t = (ctypes.c_double * n)(*[float(x) for x in times])
    fs = (ctypes.c_char_p * n)(*[os.fsencode(x) for x in files])
    _check(lib().st_write_pvd(os.fsencode(path), n, t, fs))


EXCHANGE = {"copy": 0, "mapped": 1}


def set_exchange_mode(mode):
    """"copy" (DMA copies of U and UTrans) or "mapped" (kernels use the pinned pages)."""
    _check(lib().st_set_exchange_mode(EXCHANGE[mode] if isinstance(mode, str) else mode))


def finalize():
    _check(lib().st_finalize())
