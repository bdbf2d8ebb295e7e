"""Synthetic inputs of the benchmark configurations (seeded, host-generated).

No public dataset or benchmark suite is involved; the reference itself uses random parcels
(init!/initWithHilbert!, A:504-638) and a random cell velocity in its REPL test (A:1645-1650).
These generators produce the benchmark's inputs on the host so that the GPU path and the
CPU oracle consume identical bytes:

  * fluid: U = U0 (sin(pi x/L) cos(pi y/L) cos(pi z/L), -cos(pi x/L) sin(pi y/L) cos(pi z/L), 0)
    at cell centres, optionally scaled per step by (1 + 0.2 sin(2 pi t / 0.05 s));
  * parcels: positions uniform in the box, velocity 0, diameters lognormal
    d = 20 um * exp(0.3 N(0,1)), numpy PCG64 streams seeded per configuration;
  * physics: rho_p = 1000, rho_f = 1.2 kg/m^3, nu = 1.5e-5 m^2/s (mu_f = 1.8e-5 Pa s),
    Schiller-Naumann drag, explicit Euler, dt = 1e-4 s, reflecting walls.
"""
import numpy as np

RHO_P = 1000.0
RHO_F = 1.2
NU_F = 1.5e-5
MU_F = RHO_F * NU_F
DT = 1e-4
L_BOX = 0.1

CONFIGS = {
    # 32^3 hex, 1e5 parcels, FP64, 100 steps (the CPU-runnable case)
    "hex32_fp64": dict(n=32, nparcels=100_000, seed=0, precision="fp64", steps=100,
                       U0=1.0, time_varying=False, sort_interval=0),
    # 128^3 hex, 1e7 parcels, mixed precision, 500 steps, Morton re-sort every 20 steps,
    # time-varying field
    "hex128_mixed": dict(n=128, nparcels=10_000_000, seed=0, precision="mixed", steps=500,
                         U0=1.0, time_varying=True, sort_interval=20),
    # 64 clouds, sizes log-uniform in [1e3, 2e6] (seed 2), per-cloud median diameter uniform
    # in [5, 50] um, one shared 64^3 mesh, own source per cloud, 100 steps.  Ten substeps of
    # dt/10 (the reference's nSteps): a 2 um parcel has tau_p ~ 1.2e-5 s, and explicit Euler
    # needs dt_sub / tau_p < 2
    "clouds64_hex64": dict(n=64, nclouds=64, seed=2, precision="mixed", steps=100, substeps=10,
                           size_min=1_000, size_max=2_000_000, dmed_min=5e-6, dmed_max=50e-6),
    # 96^3 hexes x 6 tets, vertices jittered +-0.15 h (seed 1), 2e7 parcels, U0 = 3 m/s,
    # mixed precision, 200 steps, face-walk relocation
    "tets96x6_mixed": dict(n=96, nparcels=20_000_000, seed=0, mesh_seed=1, jitter=0.15,
                           precision="mixed", steps=200, U0=3.0, sort_interval=10),
    # adjoint: 128^3 hex, 1e6 parcels, 200 steps, checkpoints every 20 steps; the target
    # source comes from a forward run with drag multiplier 1.1 and diameters x 0.95
    "adjoint_hex128": dict(n=128, nparcels=1_000_000, seed=3, precision="mixed", steps=200,
                           checkpoint=20, U0=1.0, time_varying=False, target_alpha=1.1,
                           target_dscale=0.95),
}


def cell_centres(n, L=L_BOX):
    h = L / n
    c = (np.arange(n) + 0.5) * h
    # cell index k*n*n + j*n + i (x fastest), A:684-691
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return x.reshape(-1), y.reshape(-1), z.reshape(-1)


def tgv_field(n, U0=1.0, L=L_BOX, dtype=np.float32):
    """Taylor-Green-like analytic field at cell centres, [n^3, 3] (cell-major AoS)."""
    x, y, z = cell_centres(n, L)
    a, b, c = np.pi * x / L, np.pi * y / L, np.pi * z / L
    U = np.empty((x.size, 3), dtype=np.float64)
    U[:, 0] = U0 * np.sin(a) * np.cos(b) * np.cos(c)
    U[:, 1] = -U0 * np.cos(a) * np.sin(b) * np.cos(c)
    U[:, 2] = 0.0
    return U.astype(dtype)


def parcels(nparcels, seed, L=L_BOX, d_median=20e-6, sigma=0.3, dtype_v=np.float32):
    """Positions uniform in [0, L)^3 (FP64), zero velocity, lognormal diameters rounded to
    the velocity precision (so that every consumer sees the same values)."""
    rng = np.random.default_rng(seed)
    xyz = rng.random((3, nparcels)) * L
    np.minimum(xyz, L * (1.0 - 1e-6), out=xyz)  # stays inside after rounding to FP32
    d = (d_median * np.exp(sigma * rng.standard_normal(nparcels))).astype(dtype_v)
    uvw = np.zeros((3, nparcels), dtype=np.float64)
    return xyz, uvw, d.astype(np.float64)


# Each hex (cube vertices numbered v0 = (0,0,0), v1 = (1,0,0), v2 = (1,1,0), v3 = (0,1,0),
# v4..v7 the same at z = 1) splits into six tetrahedra around the diagonal v0-v6; the split is
# conforming between neighbouring hexes and every tet is positively oriented.
KUHN_TETS = ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6))
CUBE = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def _morton3(i, j, k):
    def spread(v):
        v = v.astype(np.uint64) & np.uint64(0x3FF)
        v = (v | (v << np.uint64(16))) & np.uint64(0x030000FF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x0300F00F)
        v = (v | (v << np.uint64(4))) & np.uint64(0x030C30C3)
        v = (v | (v << np.uint64(2))) & np.uint64(0x09249249)
        return v
    return spread(i) | (spread(j) << np.uint64(1)) | (spread(k) << np.uint64(2))


def kuhn_tet_mesh(n, L=L_BOX, jitter=0.15, seed=1):
    """n^3 hexes on [0, L]^3, each split into 6 tets; vertices jittered uniformly by +-jitter*h
    (seeded), boundary vertices only tangentially so the walls stay planar.  Hexes are
    numbered in Morton order and tet = 6 hex + s.  Returns (vertices [nv,3] float64,
    tets [nt,4] int32, neighbours [nt,4] int32 (tet across the face opposite local vertex f,
    -1 on the boundary), hex_ijk [nhex,3])."""
    h = L / n
    g = np.arange(n + 1)
    vk, vj, vi = np.meshgrid(g, g, g, indexing="ij")
    ijk = np.stack([vi.ravel(), vj.ravel(), vk.ravel()], axis=1)
    verts = ijk.astype(np.float64) * h
    rng = np.random.default_rng(seed)
    jit = rng.uniform(-jitter * h, jitter * h, verts.shape)
    jit[(ijk == 0) | (ijk == n)] = 0.0          # walls stay planar
    verts = verts + jit
    hk, hj, hi = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    hex_ijk = np.stack([hi.ravel(), hj.ravel(), hk.ravel()], axis=1)
    order = np.argsort(_morton3(hex_ijk[:, 0], hex_ijk[:, 1], hex_ijk[:, 2]), kind="stable")
    hex_ijk = hex_ijk[order]
    nh = hex_ijk.shape[0]

    def vid(o):
        c = hex_ijk + np.array(CUBE[o])
        return (c[:, 2] * (n + 1) + c[:, 1]) * (n + 1) + c[:, 0]

    corner = np.stack([vid(o) for o in range(8)], axis=1)
    tets = np.empty((nh, 6, 4), dtype=np.int32)
    for s_, t in enumerate(KUHN_TETS):
        tets[:, s_, :] = corner[:, list(t)]
    tets = tets.reshape(-1, 4)
    nt = tets.shape[0]
    # neighbours by matching sorted face triples
    faces = np.empty((nt, 4, 3), dtype=np.int64)
    for f in range(4):
        faces[:, f, :] = np.sort(np.delete(tets, f, axis=1), axis=1)
    faces = faces.reshape(-1, 3)
    key = (faces[:, 0] * (n + 1) ** 3 + faces[:, 1]) * (n + 1) ** 3 + faces[:, 2]
    srt = np.argsort(key, kind="stable")
    ks = key[srt]
    nbr = -np.ones(nt * 4, dtype=np.int64)
    same = ks[1:] == ks[:-1]
    a, b = srt[:-1][same], srt[1:][same]
    nbr[a] = b // 4
    nbr[b] = a // 4
    return verts, tets, nbr.reshape(nt, 4).astype(np.int32), hex_ijk


def tet_centroids(verts, tets):
    return verts[tets].mean(axis=1)


def tgv_at(points, U0=1.0, L=L_BOX, dtype=np.float32):
    """The Taylor-Green-like field evaluated at given points [m, 3] (tet centroids)."""
    a, b, c = (np.pi * points[:, k] / L for k in range(3))
    U = np.empty((points.shape[0], 3), dtype=np.float64)
    U[:, 0] = U0 * np.sin(a) * np.cos(b) * np.cos(c)
    U[:, 1] = -U0 * np.cos(a) * np.sin(b) * np.cos(c)
    U[:, 2] = 0.0
    return U.astype(dtype)


def tet_hints(xyz, hex_ijk, n, L=L_BOX):
    """A starting tet for each parcel: the first tet of the hex of the unjittered lattice."""
    h = L / n
    ijk = np.clip(np.floor(xyz / h).astype(np.int64), 0, n - 1)
    rank = np.empty(n ** 3, dtype=np.int64)
    lin = (hex_ijk[:, 2] * n + hex_ijk[:, 1]) * n + hex_ijk[:, 0]
    rank[lin] = np.arange(hex_ijk.shape[0])
    hx = rank[(ijk[2] * n + ijk[1]) * n + ijk[0]]
    return (6 * hx).astype(np.int32)


def cloud_sizes(cfg):
    """Cloud sizes log-uniform in [size_min, size_max] and per-cloud median diameters."""
    rng = np.random.default_rng(cfg["seed"])
    sizes = np.exp(rng.uniform(np.log(cfg["size_min"]), np.log(cfg["size_max"]),
                               cfg["nclouds"])).astype(np.int64)
    dmed = rng.uniform(cfg["dmed_min"], cfg["dmed_max"], cfg["nclouds"])
    return sizes, dmed


def fluid_scale(step, dt=DT, time_varying=True):
    """(1 + 0.2 sin(2 pi t / 0.05 s)) with t at the start of the step."""
    if not time_varying:
        return 1.0
    t = step * dt
    return 1.0 + 0.2 * np.sin(2.0 * np.pi * t / 0.05)


def algorithmic_bytes(precision, nparcels, ncells):
    """Compulsory HBM traffic of one step (bytes): parcel state read + written once, U read
    once and the FP64 source written once.  Per parcel: mixed 40 R + 36 W = 76 B, FP64
    56 R + 48 W = 104 B, FP32 28 R + 24 W = 52 B.  Per cell: U (12 or 24 B) + source 24 B."""
    bp = {"mixed": 76, "fp64": 104, "fp32": 52}[precision]
    bc = {"mixed": 36, "fp64": 48, "fp32": 36}[precision]
    return nparcels * bp + ncells * bc


def tet_step_kernel_bytes(precision, nparcels, ntets):
    """Compulsory traffic of the tet step kernel: the parcel state as on cuboid meshes plus
    the owning tet read and written (8 B), and once per step every tet's U (12 or 24 B), four
    FP64 face planes (128 B) and four neighbour ids (16 B); with several parcels per tet
    every tet is visited."""
    bp = {"mixed": 76, "fp64": 104}[precision] + 8
    bt = {"mixed": 12, "fp64": 24}[precision] + 128 + 16
    return nparcels * bp + ntets * bt


def step_kernel_bytes(precision, nparcels, ncells):
    """Compulsory traffic of the step kernel alone (the source write belongs to finalize)."""
    bp = {"mixed": 76, "fp64": 104, "fp32": 52}[precision]
    bu = {"mixed": 12, "fp64": 24, "fp32": 12}[precision]
    return nparcels * bp + ncells * bu
