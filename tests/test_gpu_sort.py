"""GPU tests of the periodic re-sort through the C ABI: after the set-up sort and after a
re-sort during stepping, the device-side order (st_get_order) is a permutation that groups
parcels by owning cell in key order (the Morton code of the cell on cuboid meshes up to 1024
cells per axis, the linear cell index on wider ones, the owning tet on tet meshes).  Key ranges
wider than 2^24 values are coarsened by dropping low bits (of each Morton coordinate, or of the
index or tet number), so the library's counting sort serves every mesh; the three kinds of
coarsening are covered.  Results do not depend on the order (the parity tests compare runs
with and without re-sorting)."""
import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

L = workload.L_BOX


def _params(**kw):
    kw.setdefault("precision", "mixed")
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", n_substeps=1, **kw)


def _check_grouped(order, keys_by_id):
    n = keys_by_id.shape[0]
    assert np.array_equal(np.sort(order), np.arange(n, dtype=np.int32))
    k = keys_by_id[order]
    assert np.all(k[1:] >= k[:-1])


def _morton_keys(cells, nx, ny):
    i = cells % nx
    j = (cells // nx) % ny
    k = cells // (nx * ny)
    return workload._morton3(i, j, k)


@pytest.mark.parametrize("n,prec", [(32, "mixed"), (48, "mixed"), (32, "fp32"), (32, "fp64")])
def test_cuboid_resort_groups_parcels_by_morton_key(n, prec):
    """Counting sort: 32^3 (15-bit keys) and 48^3 (18-bit keys, a Morton range wider than the
    mesh).  The carrier field is scaled by 10 so that many parcels change cell between sorts
    while every step stays shorter than a cell (the reference's relocation assumes that)."""
    m = 200000
    xyz, uvw, d = workload.parcels(m, 11)
    U = workload.tgv_field(n)
    if prec == "fp64":
        U = U.astype(np.float64)
    with st.ParcelTracker(_params(sort_interval=5, precision=prec),
                          st.mesh_desc(n, 0.0, L)) as h:
        h.set_parcels(xyz, uvw, d)
        c0 = h.get_cells()
        _check_grouped(h.get_order(), _morton_keys(c0, n, n))
        h.set_fluid_velocity(U)
        for s in range(5):                         # the re-sort runs after the fifth step
            h.step(workload.DT, 10.0)
        h.synchronize()
        c1 = h.get_cells()
        assert np.count_nonzero(c1 != c0) > m // 50
        _check_grouped(h.get_order(), _morton_keys(c1, n, n))
        for s in range(2):                         # moved on since: still a permutation
            h.step(workload.DT, 10.0)
        order = h.get_order()
        assert np.array_equal(np.sort(order), np.arange(m, dtype=np.int32))


def test_wide_mesh_sorts_by_coarsened_linear_cell():
    """1100 x 1100 x 14 cells (more than 2^24, wider than 1024): linear cell keys less their
    lowest bit (25-bit indices, 24-bit keys)."""
    dims = (1100, 1100, 14)
    m = 100000
    rng = np.random.default_rng(3)
    xyz = rng.uniform(0.0, L, (3, m))
    uvw = np.zeros((3, m))
    d = np.full(m, 2e-5)
    mesh = st.mesh_desc(dims, 0.0, L)
    with st.ParcelTracker(_params(sort_interval=3), mesh) as h:
        h.set_parcels(xyz, uvw, d)
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64) >> 1)
        h.set_fluid_velocity(np.zeros((int(np.prod(dims)), 3), np.float32))
        for s in range(3):
            h.step(workload.DT, 1.0)
        h.synchronize()
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64) >> 1)


def test_morton_keys_coarsened_above_256_cells_per_axis():
    """300 x 20 x 12 cells: 9-bit coordinates would make 27-bit Morton keys; the keys are the
    Morton codes of (i >> 1, j >> 1, k >> 1)."""
    dims = (300, 20, 12)
    m = 80000
    rng = np.random.default_rng(5)
    xyz = rng.uniform(0.0, L, (3, m))
    uvw = rng.normal(0.0, 0.5, (3, m)).astype(np.float32).astype(np.float64)
    d = np.full(m, 2e-5)
    mesh = st.mesh_desc(dims, 0.0, L)

    def keys(cells):
        i = cells % dims[0]
        j = (cells // dims[0]) % dims[1]
        k = cells // (dims[0] * dims[1])
        return workload._morton3(i >> 1, j >> 1, k >> 1)

    with st.ParcelTracker(_params(sort_interval=3), mesh) as h:
        h.set_parcels(xyz, uvw, d)
        _check_grouped(h.get_order(), keys(h.get_cells().astype(np.int64)))
        h.set_fluid_velocity(np.zeros((int(np.prod(dims)), 3), np.float32))
        for s in range(3):
            h.step(workload.DT, 1.0)
        h.synchronize()
        _check_grouped(h.get_order(), keys(h.get_cells().astype(np.int64)))


def test_tet_resort_groups_parcels_by_owning_tet():
    n, m = 10, 60000
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, L, 0.15, 1)
    xyz, _, d = workload.parcels(m, 4)
    rng = np.random.default_rng(8)
    uvw = rng.normal(0.0, 2.0, (3, m)).astype(np.float32).astype(np.float64)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=3.0)
    desc = st.tet_mesh_desc(verts, tets, nbr, 0.0, L)
    with st.ParcelTracker(_params(sort_interval=4), desc) as h:
        h.set_parcels(xyz, uvw, d, hint=workload.tet_hints(xyz, hex_ijk, n, L))
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64))
        h.set_fluid_velocity(U)
        for s in range(4):
            h.step(workload.DT, 1.0)
        h.synchronize()
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64))


@pytest.mark.slow
def test_tet_mesh_above_2p24_tets_sorts_by_coarsened_tet():
    """142^3 hexes x 6 = 17,179,728 tets (more than 2^24): owning-tet keys less their lowest
    bit (25-bit tet numbers, 24-bit keys), at set-up and after a re-sort."""
    n, m = 142, 200000
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, L, 0.15, 1)
    assert tets.shape[0] > 1 << 24
    xyz, _, d = workload.parcels(m, 4)
    rng = np.random.default_rng(9)
    uvw = rng.normal(0.0, 1.0, (3, m)).astype(np.float32).astype(np.float64)
    desc = st.tet_mesh_desc(verts, tets, nbr, 0.0, L)
    with st.ParcelTracker(_params(sort_interval=2), desc) as h:
        h.set_parcels(xyz, uvw, d, hint=workload.tet_hints(xyz, hex_ijk, n, L))
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64) >> 1)
        h.set_fluid_velocity(np.zeros((tets.shape[0], 3), np.float32))
        for s in range(2):                         # the re-sort runs after the second step
            h.step(workload.DT, 1.0)
        h.synchronize()
        _check_grouped(h.get_order(), h.get_cells().astype(np.int64) >> 1)


def test_ragged_clouds_share_the_bins():
    """Several clouds of ragged sizes (partial warps, a cloud of two) sorted one after the
    other with the handle's shared counting bins: each cloud's order groups its own parcels."""
    n = 16
    sizes = [2, 33, 1000, 5]
    prm = _params(n_clouds=len(sizes), sort_interval=3)
    with st.ParcelTracker(prm, st.mesh_desc(n, 0.0, L)) as h:
        for c, m in enumerate(sizes):
            xyz, uvw, d = workload.parcels(m, 40 + c)
            h.set_parcels(xyz, uvw, d, cloud=c)
        for c in range(len(sizes)):
            _check_grouped(h.get_order(c), _morton_keys(h.get_cells(c), n, n))
        h.set_fluid_velocity(workload.tgv_field(n))
        for s in range(3):
            h.step(workload.DT, 10.0)
        h.synchronize()
        for c in range(len(sizes)):
            _check_grouped(h.get_order(c), _morton_keys(h.get_cells(c), n, n))
