"""GPU test of st_step_noalloc, the step for callers that cannot allocate device memory.

Such callers (a host that gives all device memory to its own pool, or a plugin that must not
grow the process's device footprint after set-up) pass every array themselves; the library's
only scratch is a fixed-size device array.  The test drives it through the C ABI on arrays
that the test allocates itself (with torch), twice in a row, and checks each call against
st_step on a handle: positions and velocities bit-identical, source within the one-limb
fixed-point tolerance of the other GPU tests.  This file is collected last."""
import ctypes

import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

TOL_SRC_1LIMB = 1e-8


def relerr(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def _params():
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision="mixed", n_substeps=1)


def test_step_noalloc_matches_st_step_on_two_calls():
    import torch

    n, npcl = 32, 60000
    xyz, uvw, d = workload.parcels(npcl, 21)
    U = workload.tgv_field(n, dtype=np.float32)
    prm = _params()
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    fs = [workload.fluid_scale(k) for k in range(2)]

    ref = []
    with st.ParcelTracker(prm, mesh) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(2):
            h.step(workload.DT, fs[k])
            h.synchronize()
            px, pu, _ = h.get_parcels()
            ref.append((px, pu, h.get_source()))

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    X = [torch.tensor(xyz[a], dtype=torch.float64, device=dev) for a in range(3)]
    V = [torch.tensor(uvw[a], dtype=torch.float32, device=dev) for a in range(3)]
    D = torch.tensor(d, dtype=torch.float32, device=dev)
    Ud = torch.tensor(U.reshape(-1), device=dev)
    S = torch.full((n ** 3 * 3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k in range(2):
        rc = st.lib().st_step_noalloc(ctypes.byref(prm), ctypes.byref(mesh), npcl,
                                      X[0].data_ptr(), X[1].data_ptr(), X[2].data_ptr(),
                                      V[0].data_ptr(), V[1].data_ptr(), V[2].data_ptr(),
                                      D.data_ptr(), Ud.data_ptr(), S.data_ptr(), workload.DT,
                                      fs[k], stream)
        assert rc == st.ST_OK, st.last_error()
        torch.cuda.synchronize()
        px = np.stack([t.cpu().numpy() for t in X])
        pu = np.stack([t.cpu().numpy().astype(np.float64) for t in V])
        src = S.cpu().numpy().reshape(-1, 3)
        assert np.array_equal(px, ref[k][0]), f"positions differ after call {k + 1}"
        assert np.array_equal(pu, ref[k][1]), f"velocities differ after call {k + 1}"
        assert relerr(src, ref[k][2]) <= TOL_SRC_1LIMB, f"source differs after call {k + 1}"


def _device_arrays(torch, xyz, uvw, d, U, ncomp):
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    X = [torch.tensor(xyz[a], dtype=torch.float64, device=dev) for a in range(3)]
    V = [torch.tensor(uvw[a], dtype=torch.float32, device=dev) for a in range(3)]
    D = torch.tensor(d, dtype=torch.float32, device=dev)
    Ud = torch.tensor(U.reshape(-1), device=dev)
    S = torch.full((ncomp,), float("nan"), dtype=torch.float64, device=dev)
    return X, V, D, Ud, S


def _call(prm, mesh, npcl, X, V, D, Ud, S, fs, stream):
    return st.lib().st_step_noalloc(ctypes.byref(prm), ctypes.byref(mesh), npcl,
                                    X[0].data_ptr(), X[1].data_ptr(), X[2].data_ptr(),
                                    V[0].data_ptr(), V[1].data_ptr(), V[2].data_ptr(),
                                    D.data_ptr(), Ud.data_ptr(), S.data_ptr(), workload.DT, fs,
                                    stream)


def test_step_noalloc_three_substeps_matches_st_step():
    """Three substeps: intermediate deposits at cell crossings in the probe and in the
    deterministic pass."""
    import torch

    n, npcl = 16, 20000
    xyz, uvw, d = workload.parcels(npcl, 5)
    uvw = np.random.default_rng(6).normal(0.0, 2.0, uvw.shape).astype(np.float32).astype(np.float64)
    U = workload.tgv_field(n, U0=3.0, dtype=np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=3)
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    with st.ParcelTracker(prm, mesh) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.step(workload.DT, 1.0)
        h.synchronize()
        px, pu, _ = h.get_parcels()
        ref_src = h.get_source()
    X, V, D, Ud, S = _device_arrays(torch, xyz, uvw, d, U, n ** 3 * 3)
    rc = _call(prm, mesh, npcl, X, V, D, Ud, S, 1.0, torch.cuda.current_stream().cuda_stream)
    assert rc == st.ST_OK, st.last_error()
    torch.cuda.synchronize()
    assert np.array_equal(np.stack([t.cpu().numpy() for t in X]), px)
    assert np.array_equal(np.stack([t.cpu().numpy().astype(np.float64) for t in V]), pu)
    assert relerr(S.cpu().numpy().reshape(-1, 3), ref_src) <= TOL_SRC_1LIMB


def test_step_noalloc_reports_a_parcel_outside_and_steps_the_others():
    import torch

    n, npcl, bad = 16, 5000, 1234
    xyz, uvw, d = workload.parcels(npcl, 8)
    U = workload.tgv_field(n, dtype=np.float32)
    prm = _params()
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    keep = np.arange(npcl) != bad
    with st.ParcelTracker(prm, mesh) as h:
        h.set_parcels(xyz[:, keep], uvw[:, keep], d[keep])
        h.set_fluid_velocity(U)
        h.step(workload.DT, 1.0)
        h.synchronize()
        px, pu, _ = h.get_parcels()
        ref_src = h.get_source()
    xo = xyz.copy()
    xo[0, bad] = 2.5 * workload.L_BOX
    X, V, D, Ud, S = _device_arrays(torch, xo, uvw, d, U, n ** 3 * 3)
    rc = _call(prm, mesh, npcl, X, V, D, Ud, S, 1.0, torch.cuda.current_stream().cuda_stream)
    assert rc == st.ST_ERR_PARCEL_OUTSIDE, st.last_error()
    torch.cuda.synchronize()
    gx = np.stack([t.cpu().numpy() for t in X])
    gu = np.stack([t.cpu().numpy().astype(np.float64) for t in V])
    assert np.array_equal(gx[:, bad], xo[:, bad]) and np.array_equal(gu[:, bad], uvw[:, bad])
    assert np.array_equal(gx[:, keep], px)
    assert np.array_equal(gu[:, keep], pu)
    assert relerr(S.cpu().numpy().reshape(-1, 3), ref_src) <= TOL_SRC_1LIMB


def test_step_noalloc_without_parcels_gives_a_zero_source():
    import torch

    n = 8
    prm = _params()
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    U = workload.tgv_field(n, dtype=np.float32)
    e = np.zeros((3, 0))
    X, V, D, Ud, S = _device_arrays(torch, e, e, np.zeros(0), U, n ** 3 * 3)
    rc = st.lib().st_step_noalloc(ctypes.byref(prm), ctypes.byref(mesh), 0, None, None, None,
                                  None, None, None, None, Ud.data_ptr(), S.data_ptr(),
                                  workload.DT, 1.0, torch.cuda.current_stream().cuda_stream)
    assert rc == st.ST_OK, st.last_error()
    torch.cuda.synchronize()
    assert np.all(S.cpu().numpy() == 0.0)


def test_step_noalloc_refuses_a_capturing_stream():
    """The call synchronises its stream, so it refuses a stream that is being captured
    (before launching anything, so the capture stays valid)."""
    import torch

    n, npcl = 8, 1000
    xyz, uvw, d = workload.parcels(npcl, 9)
    U = workload.tgv_field(n, dtype=np.float32)
    prm = _params()
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    X, V, D, Ud, S = _device_arrays(torch, xyz, uvw, d, U, n ** 3 * 3)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc = _call(prm, mesh, npcl, X, V, D, Ud, S, 1.0, s.cuda_stream)
        g.capture_end()
    assert rc == st.ST_ERR_INVALID_ARGUMENT
    assert "captured" in st.last_error()


def test_step_noalloc_rejects_meshes_beyond_its_scratch():
    assert st.lib().st_noalloc_max_cells() == 262144
    n = 65  # 65^3 > 64^3 cells
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    rc = st.lib().st_step_noalloc(ctypes.byref(_params()), ctypes.byref(mesh), 0, None, None,
                                  None, None, None, None, None, 1, 1, workload.DT, 1.0, None)
    assert rc == st.ST_ERR_INVALID_ARGUMENT
    assert "too large" in st.last_error()
