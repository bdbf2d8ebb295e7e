"""GPU tests of the asynchronous coupling shim (st_evolve_cloud_async), the reference's default
mode: each call returns the constant extrapolation est_k = 2 S_{k-1} - est_{k-1} (est_0 = 0)
of the source, where S_{k-1} is the true source of the step the previous call launched, and
that step runs with the U given to its own call.

The true sources come from the synchronous shim (st_evolve_cloud) on the same inputs, which
the parity tests tie to the oracle; the step is deterministic, so the recursion is checked
bit for bit in FP64 and to FP32 rounding with 4-byte exchange arrays."""
import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

N, NPCL, STEPS = 24, 40000, 7


def _setup(tbytes):
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=3)
    st.setup(prm, st.mesh_desc(N, 0.0, workload.L_BOX))
    xyz, uvw, d = workload.parcels(NPCL, 21)
    h = st.default_handle()
    assert st.lib().st_set_parcels(h, 0, NPCL, xyz.ctypes.data, uvw.ctypes.data,
                                   d.ctypes.data) == 0
    U = st.allocate_array("U", N ** 3, 3, tbytes)
    UT = st.allocate_array("UTrans", N ** 3, 3, tbytes)
    return U, UT


def _fields():
    base = workload.tgv_field(N).astype(np.float64)
    return [base * workload.fluid_scale(k, workload.DT, True) for k in range(STEPS)]


def _true_sources(tbytes):
    """S_k of the synchronous shim for the same U sequence."""
    U, UT = _setup(tbytes)
    try:
        out = []
        for Uk in _fields():
            U[:] = Uk
            st.evolve_cloud(workload.DT)
            out.append(UT.astype(np.float64).copy())
        return out
    finally:
        st.finalize()


def _async_outputs(tbytes):
    U, UT = _setup(tbytes)
    try:
        out = []
        for Uk in _fields():
            U[:] = Uk
            st.evolve_cloud_async(workload.DT)
            out.append(UT.astype(np.float64).copy())
        return out
    finally:
        st.finalize()


def test_async_coupling_is_constant_extrapolation_fp64():
    S = _true_sources(8)
    E = _async_outputs(8)
    est = np.zeros_like(S[0])
    assert np.array_equal(E[0], est)                      # est_0 = 0
    for k in range(1, STEPS):
        est = 2.0 * S[k - 1] - est
        assert np.array_equal(E[k], est), k
    assert np.abs(S[-1]).max() > 0


def test_async_coupling_with_float_exchange_arrays():
    S = _true_sources(8)                                  # FP64 true sources
    E = _async_outputs(4)
    est = np.zeros_like(S[0])
    for k in range(1, STEPS):
        est = 2.0 * S[k - 1] - est
        assert np.array_equal(E[k], est.astype(np.float32).astype(np.float64)), k


def test_async_then_finalize_and_setup_again():
    """A step still running at st_finalize or at a new st_setup is drained first."""
    for _ in range(2):
        U, UT = _setup(4)
        U[:] = workload.tgv_field(N)
        st.evolve_cloud_async(workload.DT)
        st.evolve_cloud_async(workload.DT)
    st.finalize()


@pytest.mark.parametrize("tbytes", [4, 8])
def test_mapped_exchange_equals_copies(tbytes):
    """Zero-copy exchange (kernels use the pinned U / UTrans pages) gives the same UTrans as
    the DMA copies, step after step."""
    ref = _true_sources(tbytes)
    U, UT = _setup(tbytes)
    try:
        st.set_exchange_mode("mapped")
        for k, Uk in enumerate(_fields()):
            U[:] = Uk
            st.evolve_cloud(workload.DT)
            assert np.array_equal(UT.astype(np.float64), ref[k]), k
    finally:
        st.finalize()


def test_setup_with_another_mesh_rejects_old_exchange_arrays():
    """st_setup on a different mesh keeps the arrays the caller holds; a step then refuses
    them (instead of copying past their end) until st_finalize releases them."""
    U, UT = _setup(4)
    try:
        prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                        precision="mixed")
        st.setup(prm, st.mesh_desc(2 * N, 0.0, workload.L_BOX))
        for call in (st.evolve_cloud, st.evolve_cloud_async):
            with pytest.raises(st.ScaleTrackError) as ei:
                call(workload.DT)
            assert ei.value.code == st.ST_ERR_INVALID_ARGUMENT
            assert "st_finalize" in str(ei.value)
    finally:
        st.finalize()
    _setup(4)                      # a fresh allocation after st_finalize works again
    st.finalize()


@pytest.mark.parametrize("mode", ["copy", "mapped"])
@pytest.mark.parametrize("tbytes", [4, 8])
def test_sync_shim_with_overlapped_finalize_turned_on(tbytes, mode):
    """The shims' default handle converts each step's source in line; a caller may turn the
    overlapped conversion on for it (st_set_finalize_overlap), and st_evolve_cloud must then
    still hand out each step's own source, in both exchange modes."""
    ref = _true_sources(tbytes)
    U, UT = _setup(tbytes)
    try:
        st.set_exchange_mode(mode)
        assert st.lib().st_set_finalize_overlap(st.default_handle(), 1) == 0
        for k, Uk in enumerate(_fields()):
            U[:] = Uk
            st.evolve_cloud(workload.DT)
            assert np.array_equal(UT.astype(np.float64), ref[k]), f"step {k}"
    finally:
        st.finalize()


def test_async_shim_with_overlapped_finalize_turned_on():
    ref = _async_outputs(8)
    U, UT = _setup(8)
    try:
        assert st.lib().st_set_finalize_overlap(st.default_handle(), 1) == 0
        for k, Uk in enumerate(_fields()):
            U[:] = Uk
            st.evolve_cloud_async(workload.DT)
            assert np.array_equal(UT.astype(np.float64), ref[k]), f"call {k}"
    finally:
        st.finalize()
