"""GPU parity of the face-walk step on tetrahedral meshes, through the C ABI, against the CPU
oracle: positions, velocities and owning tets bit-exact, the deterministic fixed-point source
bit-exact with the oracle's fixed-point model, walk-length histograms equal."""
import glob
import os

import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

L = workload.L_BOX


def _setup(n, m, seed, speed, d_median, U0=3.0):
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, L, 0.15, 1)
    xyz, _, d = workload.parcels(m, seed, d_median=d_median)
    rng = np.random.default_rng(seed + 100)
    uvw = rng.normal(0.0, speed, (3, m)).astype(np.float32).astype(np.float64)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=U0)
    hint = workload.tet_hints(xyz, hex_ijk, n, L)
    return (verts, tets, nbr), xyz, uvw, d, U, hint


def _gpu(prm, mesh, xyz, uvw, d, U, hint, dt, fscales, hop_limit=0):
    desc = st.tet_mesh_desc(*mesh, 0.0, L, hop_limit=hop_limit)
    with st.ParcelTracker(prm, desc) as h:
        h.set_parcels(xyz, uvw, d, hint=hint)
        c0 = h.get_cells()
        h.set_fluid_velocity(U)
        for fs in fscales:
            h.step(dt, fs)
        h.synchronize()
        x, v, _ = h.get_parcels()
        return dict(xyz=x, uvw=v, cells=h.get_cells(), src=h.get_source(0), cells0=c0,
                    hops=h.hop_histogram())


def _oracle(prm, mesh, xyz, uvw, d, U, cells0, dt, fscales, hop_limit=64):
    cfg = oracle.make_cfg(1, 0.0, L, prm.mu_c, prm.rho_c, prm.rho_d, drag=prm.drag_model,
                          precision=prm.precision, n_substeps=prm.n_substeps,
                          quant_limbs=2 if prm.precision == 2 else 1)
    Uv = U.astype(np.float64) if prm.precision == 2 else U.astype(np.float32).astype(np.float64)
    return oracle.tet_run(cfg, mesh, xyz, uvw, d, cells0, Uv, len(fscales), dt, fscale=fscales,
                          hop_limit=hop_limit)


CASES = [
    # drag, precision, substeps, dt, initial speed, median diameter, re-sort interval
    ("stokes_implicit", "mixed", 1, 1e-3, 20.0, 20e-6, 2),
    ("schiller_naumann", "mixed", 3, 1e-3, 10.0, 40e-6, 0),
    ("stokes_implicit", "fp64", 2, 1e-3, 20.0, 20e-6, 2),
    ("schiller_naumann", "fp64", 1, 1e-4, 1.0, 20e-6, 1),
]


@pytest.mark.parametrize("drag,prec,nsub,dt,speed,dmed,sort", CASES,
                         ids=[f"{c[0]}-{c[1]}-sub{c[2]}" for c in CASES])
def test_tet_step_matches_oracle(drag, prec, nsub, dt, speed, dmed, sort):
    n, m = 8, 20000
    mesh, xyz, uvw, d, U, hint = _setup(n, m, 5, speed, dmed)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model=drag, precision=prec, n_substeps=nsub, sort_interval=sort,
                    n_clouds=1)
    fscales = [workload.fluid_scale(k) for k in range(4)]
    U_dev = U if prec == "mixed" else U.astype(np.float64)
    g = _gpu(prm, mesh, xyz, uvw, d, U_dev, hint, dt, fscales)
    cells0, status = oracle.tet_locate(mesh, xyz, hint, 1 << 20)
    assert (status == 0).all()
    assert np.array_equal(g["cells0"], cells0), "initial owning tets differ"
    r = _oracle(prm, mesh, xyz, uvw, d, U_dev, cells0, dt, fscales)
    assert r["lost"] == 0 and r["overflow"] == 0
    assert np.array_equal(g["xyz"], r["xyz"]), "positions differ"
    assert np.array_equal(g["uvw"], r["uvw"]), "velocities differ"
    assert np.array_equal(g["cells"], r["cells"]), "owning tets differ"
    assert np.array_equal(g["src"], r["src_quant"]), "fixed-point source differs"
    assert np.array_equal(g["hops"].astype(np.int64), r["hop_hist"]), (g["hops"], r["hop_hist"])
    if speed >= 10.0:
        assert r["hop_hist"][2:].sum() > 0                  # multi-hop walks were exercised
    # FP64 sum of the same deposits: within the fixed-point tolerance
    s = np.abs(r["src_seq"]).max()
    tol = 1e-14 if prec == "fp64" else 1e-8
    assert np.abs(g["src"] - r["src_seq"]).max() <= tol * s


def test_tet_set_parcels_without_hint_walks_from_tet_zero():
    n, m = 6, 3000
    mesh, xyz, uvw, d, U, hint = _setup(n, m, 11, 0.0, 20e-6)
    prm = st.params(precision="mixed", sort_interval=0)
    with st.ParcelTracker(prm, st.tet_mesh_desc(*mesh, 0.0, L)) as h:
        h.set_parcels(xyz, uvw, d)
        cells = h.get_cells()
    ref, status = oracle.tet_locate(mesh, xyz, np.zeros(m, np.int32), 1 << 20)
    assert (status == 0).all()
    assert np.array_equal(cells, ref)


def test_tet_parcel_outside_box_is_rejected():
    n = 4
    mesh, xyz, uvw, d, U, hint = _setup(n, 100, 12, 0.0, 20e-6)
    xyz[0, 7] = 1.5 * L
    prm = st.params(precision="mixed")
    with st.ParcelTracker(prm, st.tet_mesh_desc(*mesh, 0.0, L)) as h:
        with pytest.raises(st.ScaleTrackError) as e:
            h.set_parcels(xyz, uvw, d, hint=hint)
        assert e.value.code == st.ST_ERR_PARCEL_OUTSIDE


def test_tet_hop_limit_loses_parcels_and_reports_them():
    """A hop limit of 1 with fast parcels: the lost parcels are counted as by the oracle and
    the step reports ST_ERR_PARCEL_OUTSIDE on the next synchronisation."""
    n, m = 8, 5000
    mesh, xyz, uvw, d, U, hint = _setup(n, m, 13, 30.0, 20e-6)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="stokes_implicit", precision="mixed", n_substeps=1)
    cells0, _ = oracle.tet_locate(mesh, xyz, hint, 1 << 20)
    r = _oracle(prm, mesh, xyz, uvw, d, U, cells0, 1e-3, [1.0], hop_limit=1)
    assert r["lost"] > 0
    with st.ParcelTracker(prm, st.tet_mesh_desc(*mesh, 0.0, L, hop_limit=1)) as h:
        h.set_parcels(xyz, uvw, d, hint=hint)
        h.set_fluid_velocity(U)
        h.step(1e-3, 1.0)
        with pytest.raises(st.ScaleTrackError) as e:
            h.synchronize()
        assert e.value.code == st.ST_ERR_PARCEL_OUTSIDE
        assert str(r["lost"]) in str(e.value)
        x, v, _ = h.get_parcels(check=False)
    assert np.array_equal(x, r["xyz"]) and np.array_equal(v, r["uvw"])


def test_tet_graph_replay_equals_steps():
    n, m = 8, 20000
    mesh, xyz, uvw, d, U, hint = _setup(n, m, 14, 5.0, 20e-6)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=2)
    fs = [workload.fluid_scale(k) for k in range(6)]
    ref = _gpu(prm, mesh, xyz, uvw, d, U, hint, 1e-4, fs)
    with st.ParcelTracker(prm, st.tet_mesh_desc(*mesh, 0.0, L)) as h:
        h.set_parcels(xyz, uvw, d, hint=hint)
        h.set_fluid_velocity(U)
        h.step(1e-4, fs[0])                      # first step: probe and scale
        h.step(1e-4, fs[1])                      # re-sort after this one
        h.graph_capture(4, 1e-4, fs[2:])        # a multiple of 2 x sort_interval
        h.graph_launch()
        h.synchronize()
        x, v, _ = h.get_parcels()
        assert np.array_equal(x, ref["xyz"]) and np.array_equal(v, ref["uvw"])
        assert np.array_equal(h.get_cells(), ref["cells"])
        assert np.array_equal(h.get_source(0), ref["src"])


@pytest.mark.slow
def test_tet_full_mesh_subsample():
    """The 96^3 x 6 jittered mesh with U0 = 3 at the benchmark's time step, 1e6 parcels."""
    cfg = workload.CONFIGS["tets96x6_mixed"]
    n, m = cfg["n"], 1_000_000
    mesh, xyz, uvw, d, U, hint = _setup(n, m, cfg["seed"], 0.0, 20e-6, U0=cfg["U0"])
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=2)
    fs = [workload.fluid_scale(k) for k in range(3)]
    g = _gpu(prm, mesh, xyz, uvw, d, U, hint, workload.DT, fs)
    r = _oracle(prm, mesh, xyz, uvw, d, U, g["cells0"], workload.DT, fs)
    assert r["lost"] == 0
    assert np.array_equal(g["xyz"], r["xyz"])
    assert np.array_equal(g["uvw"], r["uvw"])
    assert np.array_equal(g["cells"], r["cells"])
    assert np.array_equal(g["src"], r["src_quant"])


TET_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                           "tet", "*.npz")))


@pytest.mark.parametrize("path", TET_GOLDEN, ids=[os.path.basename(p) for p in TET_GOLDEN])
def test_tet_step_matches_golden(path):
    """The tet fixtures of the independent Python restatement (tests/golden/gen_golden.py):
    start tets located from the hints, then positions, velocities, owning tets, the
    fixed-point source and the walk-length histogram after the fixture's steps."""
    z = np.load(path)
    n, nsub, drag, nsteps = [int(v) for v in z["meta"]]
    Lb, mu, rc, rd, dt = [float(v) for v in z["phys"]]
    prm = st.params(mu_c=mu, rho_c=rc, rho_d=rd, drag_model=drag,
                    precision=str(z["precision"]), n_substeps=nsub)
    desc = st.tet_mesh_desc(z["verts"], z["tets"], z["nbr"], 0.0, Lb)
    with st.ParcelTracker(prm, desc) as h:
        h.set_parcels(z["xyz0"], z["uvw0"].astype(np.float64), z["d"].astype(np.float64),
                      hint=z["hint"])
        assert np.array_equal(h.get_cells(), z["cells0"])
        h.set_fluid_velocity(z["U"])
        for fs in z["fscale"]:
            h.step(dt, float(fs))
        h.synchronize()
        x, v, _ = h.get_parcels()
        assert np.array_equal(x, z["xyz"])
        assert np.array_equal(v.astype(z["uvw"].dtype), z["uvw"])
        assert np.array_equal(h.get_cells(), z["cells"])
        assert np.array_equal(h.get_source(0), z["src_quant"])
        assert np.array_equal(h.hop_histogram(), z["hop_hist"])
