"""Mixed precision against the all-FP64 step at the full 128^3 x 1e7 size of the benchmark.

The source error of the mixed step is stated in three norms, each relative to the FP64
step's source S on the same inputs:
  * max-norm   max_c |S_mixed - S| / max_c |S|;
  * L2         |S_mixed - S|_2 / |S|_2;
  * per cell   |S_mixed,c - S_c| / |S_c| over the cells with |S_c| >= 1e-3 max |S|.
"One step from identical state" isolates the arithmetic: both precisions start from the same
parcels (the mixed run's state after 20 steps, so that the parcels have relaxed towards the
carrier, where FP32 cancellation would show) and take one step: the bar holds there in
every norm.  After 20 steps from the same inputs the trajectories may also have parted, and
the bar is asserted in L2 and at the 99th percentile of the per-cell error."""
import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 1e-5          # the bar on the mixed-precision momentum source
N = 128
NPCL = 10_000_000
RELAX_STEPS = 20


def params(prec):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision=prec, n_substeps=1,
                     sort_interval=20)


def source_errors(Sm, Sd):
    mx = np.abs(Sd).max()
    err = np.abs(Sm - Sd)
    sel = np.abs(Sd) >= 1e-3 * mx
    rel = err[sel] / np.abs(Sd[sel])
    return {"max": float(err.max() / mx),
            "l2": float(np.linalg.norm(Sm - Sd) / np.linalg.norm(Sd)),
            "cell_p99": float(np.percentile(rel, 99)), "cell_max": float(rel.max())}


def one_step(prec, xyz, uvw, d, U, k):
    with st.ParcelTracker(params(prec), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U.astype(np.float64 if prec == "fp64" else np.float32))
        h.step(workload.DT, workload.fluid_scale(k))
        h.synchronize()
        return h.get_source(), h.get_cells()


def test_mixed_source_one_step_from_identical_state_full_size():
    xyz, uvw, d = workload.parcels(NPCL, 0)
    U = workload.tgv_field(N, dtype=np.float32)
    with st.ParcelTracker(params("mixed"), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(RELAX_STEPS):
            h.step(workload.DT, workload.fluid_scale(k))
        h.synchronize()
        x1, u1, _ = h.get_parcels()
    Sm, cm = one_step("mixed", x1, u1, d, U, RELAX_STEPS)
    Sd, cd = one_step("fp64", x1, u1, d, U, RELAX_STEPS)
    e = source_errors(Sm, Sd)
    assert np.array_equal(cm, cd), "owning cells differ after one step from the same state"
    assert e["max"] <= TOL, e
    assert e["l2"] <= TOL, e
    assert e["cell_p99"] <= TOL, e


def test_mixed_source_after_twenty_steps_full_size():
    xyz, uvw, d = workload.parcels(NPCL, 0)
    U = workload.tgv_field(N, dtype=np.float32)
    S = {}
    for prec in ("mixed", "fp64"):
        with st.ParcelTracker(params(prec), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
            h.set_parcels(xyz, uvw, d)
            h.set_fluid_velocity(U.astype(np.float64 if prec == "fp64" else np.float32))
            for k in range(RELAX_STEPS):
                h.step(workload.DT, workload.fluid_scale(k))
            h.synchronize()
            S[prec] = h.get_source()
    e = source_errors(S["mixed"], S["fp64"])
    # After 20 steps the trajectories may have parted: a parcel that ends a step within
    # ~1e-11 m of a face can sample the neighbouring cell's U in one precision and not the
    # other, which moves its own cell's value by up to ~1e-4 of the largest (the max-norm).
    # The bar holds in L2 and per cell at the 99th percentile.
    assert e["l2"] <= TOL, e
    assert e["cell_p99"] <= TOL, e
