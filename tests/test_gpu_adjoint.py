"""GPU tests of the adjoint of the time-averaged source (the method of the 128^3, 1e6-parcel
adjoint benchmark).

The pull-back is checked (a) against the CPU adjoint of the same precision mode: the mean
source and the per-parcel velocity cotangents bit for bit, the parameter gradients to FP64
summation order; and (b) against central finite differences (h = 1e-6) of the all-FP64 CPU
objective with ownership frozen to its own forward pass, within 1e-4."""
import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

N, NPCL, T, C = 16, 3000, 30, 7


def inputs():
    xyz, uvw, d = workload.parcels(NPCL, 3)
    return xyz, uvw, d


def gpu_params(prec, alpha=1.0, s=1.0, sort_interval=0):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision=prec, n_substeps=1,
                     drag_multiplier=alpha, diameter_scale=s, sort_interval=sort_interval)


def ocfg(prec, alpha=1.0, s=1.0):
    return oracle.make_cfg(N, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                           workload.RHO_P, drag="sn_explicit", precision=prec, n_substeps=1,
                           drag_multiplier=alpha, diameter_scale=s)


def gpu_adjoint(prec, xyz, uvw, d, U, fs, cot_fn, sort_interval=0):
    with st.ParcelTracker(gpu_params(prec, sort_interval=sort_interval),
                          st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        S = h.mean_source_forward(T, C, workload.DT, fs)
        cot = cot_fn(S)
        da, ds, dv0 = h.mean_source_pullback(cot, T, C, workload.DT, fs)
        xyz2, uvw2, _ = h.get_parcels()
        assert np.array_equal(xyz2, xyz.astype(np.float64)) or prec == "fp32"
    return S, cot, da, ds, dv0


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_adjoint_matches_cpu_adjoint(prec):
    xyz, uvw, d = inputs()
    U = workload.tgv_field(N, dtype=np.float64 if prec == "fp64" else np.float32)
    fs = np.array([workload.fluid_scale(k) for k in range(T)])
    limbs = 2 if prec == "fp64" else 1
    tgt = oracle.adjoint(ocfg(prec, 1.1, 0.95), xyz, uvw, d, U, T, workload.DT, fscale=fs,
                         grad=False, mean_limbs=limbs)["mean_src"]
    S, cot, da, ds, dv0 = gpu_adjoint(prec, xyz, uvw, d, U, fs, lambda S: 2.0 * (S - tgt))
    r = oracle.adjoint(ocfg(prec), xyz, uvw, d, U, T, workload.DT, fscale=fs, cotangent=cot,
                       mean_limbs=limbs)
    assert r["status"] == 0
    assert np.array_equal(S, r["mean_src"]), "mean source differs from the CPU model"
    assert np.array_equal(dv0, r["dv0"]), "velocity cotangents differ"
    assert abs(da - r["dalpha"]) <= 1e-12 * abs(r["dalpha"])
    assert abs(ds - r["dscale"]) <= 1e-12 * abs(r["dscale"])
    assert np.abs(dv0).max() > 0 and da != 0 and ds != 0


def test_adjoint_independent_of_parcel_order():
    xyz, uvw, d = inputs()
    U = workload.tgv_field(N, dtype=np.float32)
    cot = np.random.default_rng(5).standard_normal((N ** 3, 3)) * 1e-12
    a = gpu_adjoint("mixed", xyz, uvw, d, U, None, lambda S: cot)
    b = gpu_adjoint("mixed", xyz, uvw, d, U, None, lambda S: cot, sort_interval=3)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[4], b[4])
    assert abs(a[2] - b[2]) <= 1e-12 * abs(a[2]) and abs(a[3] - b[3]) <= 1e-12 * abs(a[3])


def test_adjoint_against_finite_differences():
    """Mixed-precision GPU gradient vs central FD of the FP64 objective J = |Sbar - S*|^2
    with ownership frozen, h = 1e-6: within 1e-4 relative."""
    xyz, uvw, d = inputs()
    U64 = workload.tgv_field(N, dtype=np.float64)
    U32 = U64.astype(np.float32)
    fs = np.array([workload.fluid_scale(k) for k in range(T)])
    tgt = oracle.adjoint(ocfg("fp64", 1.1, 0.95), xyz, uvw, d, U64, T, workload.DT, fscale=fs,
                         grad=False, mean_limbs=2)["mean_src"]
    S, cot, da, ds, dv0 = gpu_adjoint("mixed", xyz, uvw, d, U32, fs, lambda S: 2.0 * (S - tgt))
    base = oracle.adjoint(ocfg("fp64"), xyz, uvw, d, U64, T, workload.DT, fscale=fs,
                          target=tgt, mean_limbs=2, grad=False)
    h = 1e-6

    def J(cfg, uv=uvw):
        return oracle.adjoint(cfg, xyz, uv, d, U64, T, workload.DT, fscale=fs, target=tgt,
                              mean_limbs=2, grad=False, frozen=base["frozen"])["J"]

    fd_a = (J(ocfg("fp64", 1 + h)) - J(ocfg("fp64", 1 - h))) / (2 * h)
    fd_s = (J(ocfg("fp64", 1.0, 1 + h)) - J(ocfg("fp64", 1.0, 1 - h))) / (2 * h)
    assert abs(da - fd_a) <= 1e-4 * abs(fd_a), (da, fd_a)
    assert abs(ds - fd_s) <= 1e-4 * abs(fd_s), (ds, fd_s)
    scale = np.abs(dv0).max()
    for i in (0, 17, 1234, 2999):
        for c in (0, 1):
            up = uvw.copy()
            up[c, i] += h
            um = uvw.copy()
            um[c, i] -= h
            fd = (J(ocfg("fp64"), up) - J(ocfg("fp64"), um)) / (2 * h)
            assert abs(dv0[c, i] - fd) <= 1e-4 * scale, (i, c, dv0[c, i], fd)


def test_pullback_requires_matching_forward():
    xyz, uvw, d = inputs()
    U = workload.tgv_field(N, dtype=np.float32)
    with st.ParcelTracker(gpu_params("mixed"), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        with pytest.raises(st.ScaleTrackError):
            h.mean_source_pullback(np.zeros((N ** 3, 3)), T, C, workload.DT)
        h.mean_source_forward(T, C, workload.DT)
        with pytest.raises(st.ScaleTrackError):
            h.mean_source_pullback(np.zeros((N ** 3, 3)), T + 1, C, workload.DT)


def test_drag_parameters_as_arguments():
    """The call sequence of the Julia rrule: drag multiplier, diameter scale and initial
    velocities set on an existing handle (st_set_drag_parameters, st_set_parcels) give the
    same mean source and gradients as a handle created with them."""
    xyz, uvw, d = inputs()
    U = workload.tgv_field(N, dtype=np.float32)
    v0 = np.random.default_rng(11).standard_normal(uvw.shape).astype(np.float32) * 0.01
    cot = np.random.default_rng(12).standard_normal((N ** 3, 3)) * 1e-12
    alpha, s = 1.07, 0.96
    with st.ParcelTracker(gpu_params("mixed", alpha, s), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, v0.astype(np.float64), d)
        h.set_fluid_velocity(U)
        S_ref = h.mean_source_forward(T, C, workload.DT)
        g_ref = h.mean_source_pullback(cot, T, C, workload.DT)
    with st.ParcelTracker(gpu_params("mixed"), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.mean_source_forward(T, C, workload.DT)
        h.set_drag_parameters(alpha, s)
        with pytest.raises(st.ScaleTrackError):   # the forward of the old parameters is gone
            h.mean_source_pullback(cot, T, C, workload.DT)
        x1, _, d1 = h.get_parcels()
        h.set_parcels(x1, v0.astype(np.float64), d1)
        S = h.mean_source_forward(T, C, workload.DT)
        g = h.mean_source_pullback(cot, T, C, workload.DT)
        with pytest.raises(st.ScaleTrackError):
            h.set_drag_parameters(0.0, 1.0)
    assert np.array_equal(S, S_ref)
    assert g[0] == g_ref[0] and g[1] == g_ref[1]
    assert np.array_equal(g[2], g_ref[2])
