"""CPU checks of the tetrahedral-mesh oracle and of the mesh generator it is run on.

The face walk has no counterpart in the reference, so it is pinned two ways: containment of
every located point is checked with barycentric coordinates computed independently in numpy,
and under a uniform carrier velocity (where the mesh cannot matter) the tet step must give the
same parcel states and the same total source as the cuboid-mesh oracle, which is itself pinned
to the reference's golden vectors."""
import ctypes
import glob
import os

import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

L = workload.L_BOX


def _mesh(n, jitter=0.15, seed=1):
    return workload.kuhn_tet_mesh(n, L, jitter, seed)


def _barycentric(verts, tets, t, x):
    """Barycentric coordinates of points x [m, 3] in tets t [m] (numpy solve)."""
    v = verts[tets[t]]                      # [m, 4, 3]
    A = np.transpose(v[:, 1:, :] - v[:, :1, :], (0, 2, 1))
    lam = np.linalg.solve(A, (x - v[:, 0, :])[..., None])[..., 0]
    return np.concatenate([1.0 - lam.sum(axis=1, keepdims=True), lam], axis=1)


def test_kuhn_mesh_is_conforming():
    n = 5
    verts, tets, nbr, hex_ijk = _mesh(n)
    nt = tets.shape[0]
    assert nt == 6 * n ** 3
    v = verts[tets]
    vol = np.einsum("ij,ij->i", np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), v[:, 3] - v[:, 0]) / 6
    assert (vol > 0).all()                                  # positively oriented, none flat
    assert abs(vol.sum() - L ** 3) <= 1e-12 * L ** 3         # fills the box
    # neighbour relation is symmetric and the shared face has the same three vertices
    for t in range(nt):
        for f in range(4):
            u = nbr[t, f]
            if u < 0:
                continue
            assert t in nbr[u]
            g = int(np.where(nbr[u] == t)[0][0])
            assert set(np.delete(tets[t], f)) == set(np.delete(tets[u], g))
    assert (nbr < 0).sum() == 12 * n * n                     # two triangles per wall square
    # boundary vertices only move along the wall
    on_wall = np.isclose(verts, 0.0) | np.isclose(verts, L)
    assert on_wall.any(axis=1).sum() == (n + 1) ** 3 - (n - 1) ** 3


def test_oracle_walk_finds_containing_tet():
    n = 6
    verts, tets, nbr, hex_ijk = _mesh(n)
    rng = np.random.default_rng(4)
    m = 4000
    x = rng.random((3, m)) * L
    hint = workload.tet_hints(x, hex_ijk, n, L)
    cells, status = oracle.tet_locate((verts, tets, nbr), x, hint)
    assert (status == 0).all()
    lam = _barycentric(verts, tets, cells, x.T)
    assert lam.min() >= -1e-9
    # from tet 0 the walk gets there too
    cells0, status0 = oracle.tet_locate((verts, tets, nbr), x, np.zeros(m, np.int32), 4096)
    assert (status0 == 0).all()
    lam0 = _barycentric(verts, tets, cells0, x.T)
    assert lam0.min() >= -1e-9


def test_walk_on_unjittered_hexes_agrees_with_floor_locate():
    """Known answer: on a uniform hex mesh split into tets (no jitter) the owning tet found by
    the face walk lies in the hex that floor-locate gives, for positions off the faces."""
    n = 7
    verts, tets, nbr, hex_ijk = _mesh(n, jitter=0.0)
    rng = np.random.default_rng(12)
    m = 20000
    x = rng.random((3, m)) * L
    h = L / n
    ijk = np.floor(x / h).astype(np.int64)
    frac = x / h - ijk
    off_faces = ((frac > 1e-9) & (frac < 1 - 1e-9)).all(axis=0)
    cells, status = oracle.tet_locate((verts, tets, nbr), x, np.zeros(m, np.int32), 4096)
    assert (status == 0).all()
    found = hex_ijk[cells // 6].T                  # (i, j, k) of the hex of each owning tet
    assert off_faces.sum() > 0.99 * m
    assert np.array_equal(found[:, off_faces], ijk[:, off_faces])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_tet_step_matches_cuboid_step_in_uniform_flow(precision):
    """Uniform U: positions, velocities and the total fixed-point source of the tet step must
    equal the cuboid step's (parcels stay clear of the walls, one substep)."""
    n = 6
    verts, tets, nbr, hex_ijk = _mesh(n)
    rng = np.random.default_rng(9)
    m = 3000
    xyz = 0.3 * L + 0.4 * L * rng.random((3, m))
    uvw = rng.normal(0.0, 1.0, (3, m))
    d = workload.parcels(m, 9, d_median=40e-6)[2]
    cfg = oracle.make_cfg(n, 0.0, L, workload.MU_F, workload.RHO_F, workload.RHO_P,
                          drag="sn_explicit", precision=precision, n_substeps=1,
                          quant_limbs=2 if precision == "fp64" else 1)
    Ut = np.tile(np.array([[0.7, -0.4, 0.25]]), (tets.shape[0], 1))
    Uh = np.tile(np.array([[0.7, -0.4, 0.25]]), (n ** 3, 1))
    if precision == "mixed":
        Ut = Ut.astype(np.float32).astype(np.float64)
        Uh = Uh.astype(np.float32).astype(np.float64)
    hint = workload.tet_hints(xyz, hex_ijk, n, L)
    cells, status = oracle.tet_locate((verts, tets, nbr), xyz, hint)
    assert (status == 0).all()
    steps, dt = 4, 2e-3
    rt = oracle.tet_run(cfg, (verts, tets, nbr), xyz, uvw, d, cells, Ut, steps, dt)
    rh = oracle.run(cfg, xyz, uvw, d, Uh, steps, dt)
    assert rt["status"] == 0 and rh["status"] == 0
    assert np.array_equal(rt["xyz"], rh["xyz"])
    assert np.array_equal(rt["uvw"], rh["uvw"])
    assert rt["scale"] == rh["scale"]
    st_, sh = rt["src_quant"].sum(axis=0), rh["src_quant"].sum(axis=0)
    if precision == "mixed":
        assert np.array_equal(st_, sh)      # one limb: per-cell values and sums are exact
    else:
        # two limbs: each per-cell value is rounded once to FP64 before this numpy sum
        assert np.abs(st_ - sh).max() <= 1e-14 * np.abs(sh).max()
    # the walk ended in the tet that contains each final position
    lam = _barycentric(verts, tets, rt["cells"], rt["xyz"].T)
    assert lam.min() >= -1e-9
    assert rt["hop_hist"][1:].sum() > 0


def test_tet_walk_hop_limit_marks_parcels_lost():
    n = 6
    verts, tets, nbr, hex_ijk = _mesh(n)
    x = np.array([[0.9 * L], [0.9 * L], [0.9 * L]])
    cells, status = oracle.tet_locate((verts, tets, nbr), x, np.zeros(1, np.int32), 3)
    assert status[0] == 2                                   # hop limit


def test_create_tet_validates_indices_on_the_host():
    """Out-of-range vertex or neighbour ids are refused before anything reaches a device."""
    verts, tets, nbr, _ = _mesh(2)
    prm = st.params(precision="mixed")
    bad = tets.copy()
    bad[3, 2] = verts.shape[0]
    h = ctypes.c_void_p()
    rc = st.lib().st_create_tet(ctypes.byref(prm),
                                ctypes.byref(st.tet_mesh_desc(verts, bad, nbr, 0.0, L)), 0,
                                ctypes.byref(h))
    assert rc == st.ST_ERR_INVALID_ARGUMENT and "vertex id" in st.last_error()
    badn = nbr.copy()
    badn[0, 0] = tets.shape[0]
    rc = st.lib().st_create_tet(ctypes.byref(prm),
                                ctypes.byref(st.tet_mesh_desc(verts, tets, badn, 0.0, L)), 0,
                                ctypes.byref(h))
    assert rc == st.ST_ERR_INVALID_ARGUMENT and "neighbour" in st.last_error()


TET_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                           "tet", "*.npz")))


def load_tet_golden(path):
    z = np.load(path)
    n, nsub, drag, nsteps = [int(v) for v in z["meta"]]
    Lb, mu, rc, rd, dt = [float(v) for v in z["phys"]]
    return z, dict(n=n, nsub=nsub, drag=drag, nsteps=nsteps, L=Lb, mu=mu, rc=rc, rd=rd, dt=dt,
                   precision=str(z["precision"]))


def test_tet_golden_fixtures_exist_in_both_precisions():
    assert {load_tet_golden(p)[1]["precision"] for p in TET_GOLDEN} == {"mixed", "fp64"}


@pytest.mark.parametrize("path", TET_GOLDEN, ids=[os.path.basename(p) for p in TET_GOLDEN])
def test_tet_oracle_matches_golden_fixture(oracle_lib, path):
    """The independent Python restatement of the face walk and the tet step
    (tests/golden/gen_golden.py): start tets, positions, velocities, owning tets, walk-length
    histogram, FP64 sum of the deposits and fixed-point source, bit for bit."""
    z, c = load_tet_golden(path)
    mesh = (z["verts"], z["tets"], z["nbr"])
    cells0, status = oracle.tet_locate(mesh, z["xyz0"], z["hint"])
    assert (status == 0).all() and np.array_equal(cells0, z["cells0"])
    cfg = oracle.make_cfg(1, 0.0, c["L"], c["mu"], c["rc"], c["rd"], drag=c["drag"],
                          precision=c["precision"], n_substeps=c["nsub"],
                          quant_limbs=2 if c["precision"] == "fp64" else 1)
    r = oracle.tet_run(cfg, mesh, z["xyz0"], z["uvw0"], z["d"], z["cells0"], z["U"],
                       c["nsteps"], c["dt"], fscale=z["fscale"])
    assert r["status"] == 0 and r["lost"] == 0 and r["overflow"] == 0
    assert np.array_equal(r["xyz"], z["xyz"])
    assert np.array_equal(r["uvw"].astype(z["uvw"].dtype), z["uvw"])
    assert np.array_equal(r["cells"], z["cells"])
    assert np.array_equal(r["hop_hist"], z["hop_hist"])
    assert np.array_equal(r["src_seq"], z["src_f64"])
    assert np.array_equal(r["src_quant"], z["src_quant"])
