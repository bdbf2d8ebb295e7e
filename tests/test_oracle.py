"""CPU tests of the oracle: pinned against the golden fixtures of the independent Python
restatement (tests/golden/gen_golden.py) in all three precision modes (FP32 reference mode,
mixed, FP64) and against analytic known answers."""
import glob
import os

import numpy as np
import pytest

import oracle
import workload

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load_golden(path):
    z = np.load(path)
    n, nsub, drag, nsteps = [int(v) for v in z["meta"]]
    ending, mu, rc, rd, dt = [float(v) for v in z["phys"]]
    prec = str(z["precision"]) if "precision" in z.files else "fp32"
    fscale = z["fscale"] if "fscale" in z.files else None
    return z, dict(n=n, nsub=nsub, drag=drag, nsteps=nsteps, ending=ending, mu=mu, rc=rc,
                   rd=rd, dt=dt, precision=prec, fscale=fscale)


def test_golden_fixtures_cover_every_precision_mode():
    precs = {load_golden(p)[1]["precision"] for p in GOLDEN}
    assert precs == {"fp32", "mixed", "fp64"}


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_matches_golden_fixture(oracle_lib, path):
    z, c = load_golden(path)
    prec = c["precision"]
    cfg = oracle.make_cfg(c["n"], 0.0, c["ending"], c["mu"], c["rc"], c["rd"], drag=c["drag"],
                          precision=prec, n_substeps=c["nsub"],
                          quant_limbs=2 if prec == "fp64" else 1)
    r = oracle.run(cfg, z["xyz0"], z["uvw0"], z["d"], z["U"], c["nsteps"], c["dt"],
                   fscale=c["fscale"])
    assert r["status"] == 0
    # positions in the position type, velocities in the velocity type: bit for bit
    assert np.array_equal(r["xyz"].astype(z["xyz"].dtype), z["xyz"])
    assert np.array_equal(r["uvw"].astype(z["uvw"].dtype), z["uvw"])
    assert np.array_equal(r["cells"], z["cells"])
    # FP64 sum of the deposits in parcel order: same order, same bits
    assert np.array_equal(r["src_seq"], z["src_f64"])
    # the deterministic fixed-point source (scale from the previous step's largest deposit)
    assert np.array_equal(r["src_quant"], z["src_quant"])
    if "src_f32" in z.files:
        # the reference's own Float32 accumulation (A:706) agrees to float rounding
        ref32 = z["src_f32"].astype(np.float64)
        scale = np.abs(z["src_f64"]).max()
        assert np.abs(ref32 - r["src_seq"]).max() <= 1e-5 * scale


def test_golden_fixtures_exercise_walls_and_crossings():
    for path in GOLDEN:
        z, c = load_golden(path)
        cfg = oracle.make_cfg(c["n"], 0.0, c["ending"], c["mu"], c["rc"], c["rd"],
                              precision=c["precision"])
        c0 = oracle.locate(cfg, z["xyz0"].astype(np.float64))
        assert np.sum(c0 != z["cells"]) >= 10, path
        assert np.abs(z["src_f64"]).max() > 0


def _single(U, xyz, uvw, d, n=4, L=1.0, mu=1e-3, rc=1e3, rd=1.0, drag="stokes_implicit",
            prec="fp64", nsub=10, dt=1e-3, nsteps=1, fscale=None):
    cfg = oracle.make_cfg(n, 0.0, L, mu, rc, rd, drag=drag, precision=prec, n_substeps=nsub,
                          quant_limbs=2 if prec == "fp64" else 1)
    Uc = np.tile(np.asarray(U, dtype=np.float64), (n ** 3, 1))
    return oracle.run(cfg, np.asarray(xyz, float).reshape(3, -1),
                      np.asarray(uvw, float).reshape(3, -1), np.atleast_1d(d), Uc, nsteps, dt,
                      fscale=fscale)


def test_stokes_implicit_relaxation_known_answer(oracle_lib):
    """v_n = u + (v0 - u)(1 + f)^-n for a parcel that stays in one cell."""
    u = np.array([0.3, -0.2, 0.1])
    v0 = np.array([-0.1, 0.05, 0.2])
    d, mu, rd, dt, nsub, nsteps = 7e-3, 1e-3, 1.0, 1e-3, 10, 5
    r = _single(u, [0.6, 0.6, 0.6], v0, d, nsub=nsub, dt=dt, nsteps=nsteps)
    f = 18 * mu * (dt / nsub) / (rd * d * d)
    expect = u + (v0 - u) * (1 + f) ** (-nsub * nsteps)
    assert np.allclose(r["uvw"].ravel(), expect, rtol=1e-13, atol=0)


def test_schiller_naumann_low_re_limit(oracle_lib):
    """At Re -> 0 the correction vanishes: v' = v + f (u - v) (explicit Stokes)."""
    u = np.array([1e-9, -2e-9, 0.5e-9])
    d, mu, rd, dt = 1e-5, 1.8e-5, 1000.0, 1e-4
    r = _single(u, [0.5, 0.5, 0.5], [0, 0, 0], d, mu=mu, rc=1.2, rd=rd, drag="sn_explicit",
                nsub=1, dt=dt)
    f = 18 * mu * dt / (rd * d * d)
    assert np.allclose(r["uvw"].ravel(), f * u, rtol=1e-6)


@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("side", [0, 1])
def test_wall_bounce_known_answer(oracle_lib, axis, side):
    """A parcel that would leave through a wall keeps that position component and mirrors
    its old velocity (A:1313-1329); the wall impulse is taken out of state0 (A:731-736)."""
    n, L = 4, 1.0
    h = L / n
    xyz = np.full(3, 0.5)
    xyz[axis] = 0.5 * h if side == 0 else L - 0.5 * h
    v = np.zeros(3)
    v[axis] = -1.0 if side == 0 else 1.0
    dt = 0.3  # displacement 0.3 > h/2: crosses the wall
    # huge parcel: the drag factor is ~1e-9, velocity almost unchanged
    r = _single([0, 0, 0], xyz, v, 10.0, n=n, L=L, nsub=1, dt=dt)
    assert np.allclose(r["xyz"].ravel(), xyz, rtol=0, atol=0)
    assert r["uvw"].ravel()[axis] == -v[axis]
    assert r["cells"][0] >= 0
    assert np.abs(r["src_seq"]).max() == 0.0  # state0 - v' = (v + 2|v|) - (-v) mirrored = 0


def test_momentum_bookkeeping_no_walls(oracle_lib):
    """Sum of the cell sources = sum of m (v_start - v_end) when no parcel meets a wall."""
    rng = np.random.default_rng(5)
    npcl, n = 2000, 16
    xyz = 0.3 + 0.4 * rng.random((3, npcl))
    uvw = rng.random((3, npcl)) - 0.5
    d = 5e-3 + 5e-3 * rng.random(npcl)
    cfg = oracle.make_cfg(n, 0.0, 1.0, 1e-3, 1e3, 1.0, drag="stokes_implicit",
                          precision="fp64", n_substeps=10, quant_limbs=2)
    U = rng.random((n ** 3, 3)) * 2 - 1
    r = oracle.run(cfg, xyz, uvw, d, U, 1, 0.02)
    m = (1.0 / 1e3) * np.pi * d ** 3 / 6
    expect = np.sum(m * (uvw - r["uvw"]), axis=1)
    got = r["src_seq"].sum(axis=0)
    assert np.allclose(got, expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())


def test_pow0687_accuracy(oracle_lib):
    """exp(a ln x) in double: the error grows with |a ln x| (the rounding of the product);
    over the physical Reynolds range it stays within a few ulp."""
    x = np.concatenate([np.geomspace(1e-300, 1e300, 20001),
                        np.random.default_rng(1).random(20000) * 1e4, [1.0, 2.0, 0.5, 5e-324]])
    y = oracle.pow0687(x)
    ref = x ** 0.687
    ok = ref > 0
    rel = np.abs(y[ok] - ref[ok]) / ref[ok]
    assert np.all(rel <= 4.4e-16 * (8.0 + np.abs(0.687 * np.log(x[ok]))))
    phys = ok & (x > 1e-6) & (x < 1e6)
    assert np.max(np.abs(y[phys] - ref[phys]) / ref[phys]) < 4e-15
    assert oracle.pow0687(np.array([0.0]))[0] == 0.0
    assert np.isnan(oracle.pow0687(np.array([np.nan]))[0])
    assert np.isinf(oracle.pow0687(np.array([np.inf]))[0])
    xf = np.concatenate([np.geomspace(1e-44, 3e38, 20001),
                         np.random.default_rng(5).random(20000) * 20]).astype(np.float32)
    yf = oracle.pow0687f(xf)
    reff = (xf.astype(np.float64) ** 0.687).astype(np.float32)
    ulp = np.abs(yf.view(np.int32).astype(np.int64) - reff.view(np.int32).astype(np.int64))
    assert ulp.max() <= 2
    assert np.isnan(oracle.pow0687f(np.array([np.nan], np.float32))[0])
    assert oracle.pow0687f(np.array([np.inf, 0.0, -1.0], np.float32)).tolist() == [np.inf, 0, 0]


def _bench_case(nparcels=20000, n=16, prec="mixed", seed=3, steps=3, limbs=1):
    xyz, uvw, d = workload.parcels(nparcels, seed)
    U = workload.tgv_field(n, dtype=np.float64 if prec == "fp64" else np.float32)
    cfg = oracle.make_cfg(n, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision=prec, n_substeps=1,
                          quant_limbs=limbs)
    fs = [workload.fluid_scale(s) for s in range(steps)]
    return cfg, xyz, uvw, d, U, fs


def test_quantized_source_close_to_fp64_sum(oracle_lib):
    cfg, xyz, uvw, d, U, fs = _bench_case()
    r = oracle.run(cfg, xyz, uvw, d, U, len(fs), workload.DT, fscale=fs)
    assert r["status"] == 0 and r["overflow"] == 0
    ref = r["src_seq"]
    err = np.abs(r["src_quant"] - ref).max() / np.abs(ref).max()
    assert err < 1e-8
    cfg2, *_ = _bench_case(prec="fp64", limbs=2)
    U64 = workload.tgv_field(16, dtype=np.float64)
    r2 = oracle.run(cfg2, xyz, uvw, d, U64, len(fs), workload.DT, fscale=fs)
    err2 = np.abs(r2["src_quant"] - r2["src_seq"]).max() / np.abs(r2["src_seq"]).max()
    assert err2 < 1e-14


def test_quantized_source_independent_of_parcel_order(oracle_lib):
    cfg, xyz, uvw, d, U, fs = _bench_case(nparcels=5000)
    r1 = oracle.run(cfg, xyz, uvw, d, U, 2, workload.DT, fscale=fs[:2])
    perm = np.random.default_rng(9).permutation(d.size)
    r2 = oracle.run(cfg, xyz[:, perm], uvw[:, perm], d[perm], U, 2, workload.DT, fscale=fs[:2])
    assert np.array_equal(r1["src_quant"], r2["src_quant"])
    assert np.array_equal(r1["xyz"][:, perm], r2["xyz"])
    assert r1["scale"] == r2["scale"]


def test_parallel_oracle_matches_serial(oracle_lib):
    cfg, xyz, uvw, d, U, fs = _bench_case(nparcels=30000)
    r1 = oracle.run(cfg, xyz, uvw, d, U, 2, workload.DT, fscale=fs[:2], nthreads=1)
    r2 = oracle.run(cfg, xyz, uvw, d, U, 2, workload.DT, fscale=fs[:2], nthreads=4)
    assert np.array_equal(r1["xyz"], r2["xyz"]) and np.array_equal(r1["uvw"], r2["uvw"])
    assert np.array_equal(r1["src_quant"], r2["src_quant"])
    assert np.allclose(r1["src_seq"], r2["src_seq"], rtol=1e-12, atol=1e-30)


def test_range_check_flags_sudden_growth(oracle_lib):
    """A deposit 2^8 x larger than the previous step's largest cannot be represented; it is
    counted as an overflow instead of wrapping the integer sum."""
    cfg, xyz, uvw, d, U, fs = _bench_case(nparcels=2000)
    r = oracle.run(cfg, xyz, uvw, d, U, 2, workload.DT, fscale=[1e-6, 1.0])
    assert r["overflow"] > 0 and (r["status"] & 2)


def test_lost_parcel_left_unchanged(oracle_lib):
    cfg = oracle.make_cfg(4, 0.0, 1.0, 1e-3, 1e3, 1.0, precision="fp64", n_substeps=1)
    xyz = np.array([[0.5, 1.5], [0.5, 0.5], [0.5, 0.5]])
    uvw = np.zeros((3, 2))
    r = oracle.run(cfg, xyz, uvw, np.array([1e-3, 1e-3]), np.ones((64, 3)), 1, 1e-3)
    assert r["lost"] == 1 and (r["status"] & 1)
    assert r["xyz"][0, 1] == 1.5 and r["cells"][1] == -1


def test_golden_fixtures_are_what_their_script_makes(tmp_path):
    """The committed fixtures are exactly the output of tests/golden/gen_golden.py (regenerated
    here into a temporary folder), so none was edited by hand."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "gen_golden", os.path.join(HERE, "golden", "gen_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    gen.main(str(tmp_path), verbose=False)
    paths = GOLDEN + sorted(glob.glob(os.path.join(HERE, "golden", "tet", "*.npz")))
    assert len(paths) == 13
    for path in paths:
        a = np.load(path)
        b = np.load(os.path.join(str(tmp_path), os.path.relpath(path, os.path.join(HERE, "golden"))))
        assert set(a.files) == set(b.files), path
        for k in a.files:
            assert np.array_equal(a[k], b[k]), (path, k)
