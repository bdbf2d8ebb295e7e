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


def test_step_noalloc_rejects_meshes_beyond_its_scratch():
    assert st.lib().st_noalloc_max_cells() == 262144
    n = 65  # 65^3 > 64^3 cells
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    rc = st.lib().st_step_noalloc(ctypes.byref(_params()), ctypes.byref(mesh), 0, None, None,
                                  None, None, None, None, None, 1, 1, workload.DT, 1.0, None)
    assert rc == st.ST_ERR_INVALID_ARGUMENT
    assert "too large" in st.last_error()
