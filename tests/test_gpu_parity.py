"""GPU parity tests: the CUDA step, called through the C ABI, against the CPU oracle.

Bar: positions, velocities and owning cells bit-exact with the oracle of the same precision
mode; the deterministic source bit-exact with the oracle's fixed-point model and within a
stated tolerance of the oracle's FP64 sum; the atomic FP64 source within 1e-12 relative."""
import glob
import os

import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))

# tolerances of the deterministic source against the FP64 sum of the same deposits
TOL_SRC_1LIMB = 1e-8    # one 64-bit limb (FP32 and mixed): 2^-30 of the largest deposit
TOL_SRC_2LIMB = 1e-14   # two limbs (FP64)
TOL_SRC_ATOMIC = 1e-12  # FP64 atomics: order-dependent rounding only


def relerr(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def gpu_run(prm, n, L, clouds, U, dt, fscales, src_dtype=np.float64):
    """clouds: list of (xyz, uvw, d).  Returns per cloud (xyz, uvw, cells, source)."""
    with st.ParcelTracker(prm, st.mesh_desc(n, 0.0, L)) as h:
        for c, (xyz, uvw, d) in enumerate(clouds):
            h.set_parcels(xyz, uvw, d, cloud=c)
        h.set_fluid_velocity(U)
        for fs in fscales:
            h.step(dt, fs)
        h.synchronize()
        out = []
        for c in range(len(clouds)):
            xyz, uvw, _ = h.get_parcels(c)
            out.append((xyz, uvw, h.get_cells(c), h.get_source(c, dtype=src_dtype)))
        return out


def oracle_cfg(n, L, prm):
    return oracle.make_cfg(n, 0.0, L, prm.mu_c, prm.rho_c, prm.rho_d, drag=prm.drag_model,
                           precision=prm.precision, n_substeps=prm.n_substeps,
                           quant_limbs=2 if prm.precision == 2 else 1,
                           drag_multiplier=prm.drag_multiplier,
                           diameter_scale=prm.diameter_scale)


def check_against_oracle(prm, n, L, xyz, uvw, d, U, dt, fscales, nthreads=0):
    g = gpu_run(prm, n, L, [(xyz, uvw, d)], U, dt, fscales)[0]
    r = oracle.run(oracle_cfg(n, L, prm), xyz, uvw, d, U.astype(np.float64), len(fscales), dt,
                   fscale=fscales, nthreads=nthreads)
    assert r["status"] == 0, r
    assert np.array_equal(g[0], r["xyz"]), "positions differ"
    assert np.array_equal(g[1], r["uvw"]), "velocities differ"
    assert np.array_equal(g[2], r["cells"]), "owning cells differ"
    return g, r


# ------------------------------------------------------------------------------------------
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_step_matches_golden(path):
    """The golden fixtures of the independent Python restatement, in the fixture's precision
    mode (FP32 reference mode, mixed, FP64) and with its per-step fluid factors."""
    z = np.load(path)
    n, nsub, drag, nsteps = [int(v) for v in z["meta"]]
    ending, mu, rc, rd, dt = [float(v) for v in z["phys"]]
    prec = str(z["precision"]) if "precision" in z.files else "fp32"
    fscales = [float(v) for v in z["fscale"]] if "fscale" in z.files else [1.0] * nsteps
    prm = st.params(mu_c=mu, rho_c=rc, rho_d=rd, drag_model=drag, precision=prec,
                    n_substeps=nsub)
    g = gpu_run(prm, n, ending, [(z["xyz0"], z["uvw0"], z["d"])], z["U"], dt, fscales)[0]
    assert np.array_equal(g[0].astype(z["xyz"].dtype), z["xyz"])
    assert np.array_equal(g[1].astype(z["uvw"].dtype), z["uvw"])
    assert np.array_equal(g[2], z["cells"])
    assert relerr(g[3], z["src_f64"]) <= (TOL_SRC_2LIMB if prec == "fp64" else TOL_SRC_1LIMB)
    assert np.array_equal(g[3], z["src_quant"])
    r = oracle.run(oracle_cfg(n, ending, prm), z["xyz0"], z["uvw0"], z["d"], z["U"], nsteps, dt,
                   fscale=fscales)
    assert np.array_equal(g[3], r["src_quant"])


def bench_inputs(nparcels, n, seed, prec):
    xyz, uvw, d = workload.parcels(nparcels, seed)
    U = workload.tgv_field(n, dtype=np.float64 if prec == "fp64" else np.float32)
    return xyz, uvw, d, U


def bench_params(prec, **kw):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision=prec, n_substeps=1, **kw)


@pytest.mark.parametrize("prec", ["mixed", "fp64", "fp32"])
def test_schiller_naumann_parity_time_varying(prec):
    n, nparcels, steps = 16, 40000, 6
    xyz, uvw, d, U = bench_inputs(nparcels, n, 1, prec)
    fs = [workload.fluid_scale(s) for s in range(steps)]
    prm = bench_params(prec)
    g, r = check_against_oracle(prm, n, workload.L_BOX, xyz, uvw, d, U, workload.DT, fs)
    assert np.array_equal(g[3], r["src_quant"]), "fixed-point source differs"
    tol = TOL_SRC_2LIMB if prec == "fp64" else TOL_SRC_1LIMB
    assert relerr(g[3], r["src_seq"]) <= tol
    moved = np.sum(g[2] != oracle.locate(oracle_cfg(n, workload.L_BOX, prm), xyz))
    assert moved > nparcels // 100  # the case exercises relocation (about 1.4 % here)


def test_stokes_substeps_mixed_and_fp64():
    """Ten substeps with intermediate deposits on cell change (A:1342-1348)."""
    n = 8
    rng = np.random.default_rng(4)
    npcl = 5000
    xyz = rng.random((3, npcl)) * 0.999
    uvw = rng.random((3, npcl)) * 2 - 1
    d = 5e-3 + 5e-3 * rng.random(npcl)
    for prec in ("mixed", "fp64"):
        U = (rng.random((n ** 3, 3)) * 2 - 1).astype(np.float32 if prec == "mixed" else np.float64)
        prm = st.params(precision=prec, n_substeps=10)
        g, r = check_against_oracle(prm, n, 1.0, xyz, uvw, d, U, 0.2, [1.0, 1.0, 1.0])
        assert np.array_equal(g[3], r["src_quant"])


def test_atomic_fp64_mode():
    n, nparcels = 16, 30000
    xyz, uvw, d, U = bench_inputs(nparcels, n, 2, "fp64")
    fs = [workload.fluid_scale(s) for s in range(4)]
    prm = bench_params("fp64", deposit="atomic")
    g, r = check_against_oracle(prm, n, workload.L_BOX, xyz, uvw, d, U, workload.DT, fs)
    assert relerr(g[3], r["src_seq"]) <= TOL_SRC_ATOMIC


def test_deterministic_source_is_bitwise_reproducible():
    n, nparcels = 32, 200000
    xyz, uvw, d, U = bench_inputs(nparcels, n, 3, "mixed")
    fs = [workload.fluid_scale(s) for s in range(5)]
    a = gpu_run(bench_params("mixed"), n, workload.L_BOX, [(xyz, uvw, d)], U, workload.DT, fs)[0]
    b = gpu_run(bench_params("mixed"), n, workload.L_BOX, [(xyz, uvw, d)], U, workload.DT, fs)[0]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_morton_resort_changes_nothing_but_order():
    """Re-sorting permutes parcels; results come back in the caller's order and the
    fixed-point source does not depend on the order of the deposits."""
    n, nparcels = 32, 100000
    xyz, uvw, d, U = bench_inputs(nparcels, n, 5, "mixed")
    fs = [workload.fluid_scale(s) for s in range(7)]
    a = gpu_run(bench_params("mixed"), n, workload.L_BOX, [(xyz, uvw, d)], U, workload.DT, fs)[0]
    b = gpu_run(bench_params("mixed", sort_interval=2), n, workload.L_BOX, [(xyz, uvw, d)], U,
                workload.DT, fs)[0]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_multiple_clouds_ragged_sizes():
    """Clouds of 0, 1, 33 and 5000 parcels in one launch, each with its own source."""
    n = 12
    sizes = [0, 1, 33, 5000]
    clouds = []
    for k, m in enumerate(sizes):
        xyz, uvw, d = workload.parcels(m, 10 + k)
        clouds.append((xyz, uvw, d))
    U = workload.tgv_field(n, dtype=np.float32)
    fs = [workload.fluid_scale(s) for s in range(3)]
    prm = bench_params("mixed", n_clouds=len(sizes), sort_interval=2)
    g = gpu_run(prm, n, workload.L_BOX, clouds, U, workload.DT, fs)
    cfg = oracle_cfg(n, workload.L_BOX, prm)
    for k, (xyz, uvw, d) in enumerate(clouds):
        r = oracle.run(cfg, xyz, uvw, d, U.astype(np.float64), len(fs), workload.DT, fscale=fs)
        assert np.array_equal(g[k][0], r["xyz"])
        assert np.array_equal(g[k][2], r["cells"])
        assert np.array_equal(g[k][3], r["src_quant"]), k
        if sizes[k] == 0:
            assert not np.any(g[k][3])


@pytest.mark.parametrize("prec", ["fp32", "mixed", "fp64"])
@pytest.mark.parametrize("drag", ["stokes_implicit", "schiller_naumann"])
def test_parcels_on_faces_walls_and_corners(prec, drag):
    """Edge positions against the oracle, bit for bit: parcels exactly on interior faces
    (floor puts them in the upper cell), on the lower walls, one ulp below the upper walls,
    in the eight corner cells, with velocities that push them across faces and into walls
    along every axis, and one cell holding many parcels (one long run for the warp scan)."""
    n, L = 8, 0.1
    h = L / n
    P = np.float32 if prec == "fp32" else np.float64
    below = float(np.nextafter(P(L), P(0)))
    pts, vel = [], []
    rng = np.random.default_rng(31)
    faces = [k * h for k in range(1, n)]
    for k in range(200):                          # exactly on interior faces
        p = rng.random(3) * L * 0.999
        p[k % 3] = faces[k % len(faces)]
        pts.append(p)
        vel.append(rng.normal(0, 2.0, 3))
    for axis in range(3):                         # on and next to every wall, moving out
        for wall, v in ((0.0, -3.0), (below, 3.0)):
            for _ in range(20):
                p = rng.random(3) * L * 0.999
                p[axis] = wall
                u = rng.normal(0, 0.5, 3)
                u[axis] = v
                pts.append(p)
                vel.append(u)
    for cx in (0.01 * h, L - 0.01 * h):           # corner cells
        for cy in (0.01 * h, L - 0.01 * h):
            for cz in (0.01 * h, L - 0.01 * h):
                pts.append(np.array([cx, cy, cz]))
                vel.append(rng.normal(0, 5.0, 3))
    for _ in range(300):                          # one crowded cell
        pts.append(np.array([3.5 * h, 4.5 * h, 2.5 * h]) + rng.uniform(-0.4, 0.4, 3) * h)
        vel.append(rng.normal(0, 0.3, 3))
    xyz = np.array(pts).T.astype(P).astype(np.float64)
    uvw = np.array(vel).T.astype(np.float32).astype(np.float64)
    d = np.full(xyz.shape[1], 30e-6)
    U = workload.tgv_field(n, U0=2.0, dtype=np.float64 if prec == "fp64" else np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model=drag, precision=prec, n_substeps=3 if drag == "stokes_implicit"
                    else 1, sort_interval=1)
    g, r = check_against_oracle(prm, n, L, xyz, uvw, d, U, 2e-3, [1.0, 0.9, 1.1])
    assert np.array_equal(g[3], r["src_quant"])
    assert r["lost"] == 0


def test_empty_and_single_parcel_clouds():
    """Clouds of 0 and 1 parcels next to a normal one, through set-up, steps and read-back."""
    n = 8
    prm = bench_params("mixed", n_clouds=3, sort_interval=2)
    xyz, uvw, d, U = bench_inputs(500, n, 13, "mixed")
    clouds = [(np.zeros((3, 0)), np.zeros((3, 0)), np.zeros(0)),
              (xyz[:, :1], uvw[:, :1], d[:1]),
              (xyz, uvw, d)]
    out = gpu_run(prm, n, workload.L_BOX, clouds, U, workload.DT, [1.0, 1.0, 1.0])
    assert out[0][0].shape == (3, 0) and not out[0][3].any()
    for c in (1, 2):
        r = oracle.run(oracle_cfg(n, workload.L_BOX, prm), *clouds[c], U.astype(np.float64), 3,
                       workload.DT)
        assert np.array_equal(out[c][0], r["xyz"]) and np.array_equal(out[c][2], r["cells"])
        assert np.array_equal(out[c][3], r["src_quant"])


def test_parcel_outside_mesh_is_rejected():
    prm = st.params(precision="mixed")
    with st.ParcelTracker(prm, st.mesh_desc(4, 0.0, 1.0)) as h:
        xyz = np.array([[0.5, 1.0], [0.5, 0.5], [0.5, 0.5]])
        with pytest.raises(st.ScaleTrackError) as e:
            h.set_parcels(xyz, np.zeros((3, 2)), np.full(2, 1e-3))
        assert e.value.code == st.ST_ERR_PARCEL_OUTSIDE
        h.set_parcels(xyz[:, :1], np.zeros((3, 1)), np.full(1, 1e-3))
        h.set_fluid_velocity(np.zeros((64, 3), np.float32))
        h.step(1e-3)
        h.synchronize()


def test_range_error_is_reported():
    """A deposit far beyond the previous step's scale is reported, not wrapped."""
    n, nparcels = 8, 2000
    xyz, uvw, d, U = bench_inputs(nparcels, n, 6, "mixed")
    with st.ParcelTracker(bench_params("mixed"), st.mesh_desc(n, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.step(workload.DT, 1e-6)
        h.step(workload.DT, 1.0)
        with pytest.raises(st.ScaleTrackError) as e:
            h.synchronize()
        assert e.value.code == st.ST_ERR_SOURCE_RANGE
        h.step(workload.DT, 1.0)   # the scale has caught up: clean again
        h.synchronize()


def test_reference_shims_allocate_array_and_evolve_cloud():
    """allocate_array_ptr + evolve_cloud with the reference's float exchange arrays."""
    z = np.load(GOLDEN[0])
    n, nsub, drag, nsteps = [int(v) for v in z["meta"]]
    ending, mu, rc, rd, dt = [float(v) for v in z["phys"]]
    prm = st.params(mu_c=mu, rho_c=rc, rho_d=rd, drag_model=drag, precision="fp32",
                    n_substeps=nsub)
    st.setup(prm, st.mesh_desc(n, 0.0, ending))
    try:
        h = st.default_handle()
        assert h
        xyz0 = np.ascontiguousarray(z["xyz0"], dtype=np.float64)
        uvw0 = np.ascontiguousarray(z["uvw0"], dtype=np.float64)
        d0 = np.ascontiguousarray(z["d"], dtype=np.float64)
        assert st.lib().st_set_parcels(h, 0, d0.size, xyz0.ctypes.data, uvw0.ctypes.data,
                                       d0.ctypes.data) == 0
        U = st.allocate_array("U", n ** 3, 3, 4)
        UT = st.allocate_array("UTrans", n ** 3, 3, 4)
        with pytest.raises(st.ScaleTrackError):
            st.allocate_array("U", n ** 3 + 1, 3, 4)   # size mismatch throws (A:1454-1465)
        U[:] = z["U"]
        for _ in range(nsteps):
            st.evolve_cloud(dt)
        assert relerr(UT.astype(np.float64), z["src_f64"]) <= 1e-6
        cells = np.empty(z["d"].size, dtype=np.int32)
        assert st.lib().st_get_cells(h, 0, cells.ctypes.data) == 0
        assert np.array_equal(cells, z["cells"])
    finally:
        st.finalize()


def test_profile_counters_and_launch_count():
    n, nparcels = 16, 10000
    xyz, uvw, d, U = bench_inputs(nparcels, n, 7, "mixed")
    with st.ParcelTracker(bench_params("mixed"), st.mesh_desc(n, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.profile(True)
        c0 = h.launch_count()
        for s in range(4):
            h.step(workload.DT)
        nstep, ms = h.profile_read("step")
        nfin, _ = h.profile_read("finalize")
        assert nstep == 4 and nfin == 4 and ms > 0
        # step, next-scale and finalize per step (the finalize overlapping the next step),
        # probe + set_scale on the first step
        assert h.launch_count() - c0 == 4 * 3 + 2
        h.set_finalize_overlap(False)
        c1 = h.launch_count()
        for s in range(4):
            h.step(workload.DT)
        h.synchronize()
        assert h.launch_count() - c1 == 4 * 2   # step and finalize (with its scale update)


@pytest.mark.slow
def test_hex32_fp64_1e5_parcels_100_steps_full_run():
    """The CPU-runnable configuration in full: 32^3 cells, 1e5 parcels, FP64, 100 steps of
    Schiller-Naumann drag with a frozen field.  Positions, velocities and cells bit-exact with
    the FP64 oracle after 100 steps; the two-limb source bit-exact with its fixed-point model
    and within 1e-14 of the FP64 sum of the same deposits."""
    c = workload.CONFIGS["hex32_fp64"]
    n, nparcels, steps = c["n"], c["nparcels"], c["steps"]
    xyz, uvw, d = workload.parcels(nparcels, c["seed"], dtype_v=np.float64)
    U = workload.tgv_field(n, U0=c["U0"], dtype=np.float64)
    prm = bench_params("fp64")
    fs = [1.0] * steps
    g, r = check_against_oracle(prm, n, workload.L_BOX, xyz, uvw, d, U, workload.DT, fs,
                                nthreads=0)
    assert np.array_equal(g[3], r["src_quant"])
    assert relerr(g[3], r["src_seq"]) <= TOL_SRC_2LIMB


@pytest.mark.slow
def test_full_size_mixed_against_oracle():
    """The benchmark sizes (128^3 cells, 1e7 parcels), a few steps: bit-exact
    state and cells and fixed-point source against the (multi-threaded) oracle."""
    cfgd = workload.CONFIGS["hex128_mixed"]
    n, nparcels = cfgd["n"], cfgd["nparcels"]
    xyz, uvw, d, U = bench_inputs(nparcels, n, cfgd["seed"], "mixed")
    fs = [workload.fluid_scale(s) for s in range(3)]
    prm = bench_params("mixed", sort_interval=2)
    g, r = check_against_oracle(prm, n, workload.L_BOX, xyz, uvw, d, U, workload.DT, fs,
                                nthreads=0)
    assert np.array_equal(g[3], r["src_quant"])
    assert relerr(g[3], r["src_seq"]) <= 1e-5   # the stated bar for the mixed source
