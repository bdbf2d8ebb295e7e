"""GPU tests of the shared-memory ring step kernel (ST_STEP_KERNEL_RING) against the per-warp
kernel (ST_STEP_KERNEL_WARP): both run the same parcel arithmetic, so positions, velocities,
owning cells and the deterministic source must agree bit for bit; the FP64 atomic source adds
in a different order and agrees to 1e-12.  Sizes cover clouds smaller than one block tile
(1280 parcels in FP32 and mixed precision, 1024 in FP64), exact multiples, several tiles per
block with a ragged end, and the default
kernel is also checked against the oracle (the parity tests use it throughout)."""
import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

N = 24


def run(kind, prec, npcl, steps=3, nsub=1, deposit="deterministic", drag="schiller_naumann",
        sort_interval=2, seed=4):
    xyz, uvw, d = workload.parcels(npcl, seed)
    U = workload.tgv_field(N, U0=2.0, dtype=np.float64 if prec == "fp64" else np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model=drag, precision=prec, n_substeps=nsub, deposit=deposit,
                    sort_interval=sort_interval)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_step_kernel(kind)
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(steps):
            h.step(workload.DT, workload.fluid_scale(k))
        h.synchronize()
        x, u, _ = h.get_parcels()
        return x, u, h.get_cells(), h.get_source()


@pytest.mark.parametrize("npcl", [1, 1000, 1024, 1280, 3 * 1280, 148 * 1280 * 2 + 517])
@pytest.mark.parametrize("prec", ["mixed", "fp64", "fp32"])
def test_ring_equals_warp_kernel(prec, npcl):
    a = run("ring", prec, npcl)
    b = run("warp", prec, npcl)
    for p, q in zip(a, b):
        assert np.array_equal(p, q)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_ring_equals_warp_kernel_substeps_and_stokes(prec):
    for nsub, drag in ((3, "schiller_naumann"), (10, "stokes_implicit")):
        a = run("ring", prec, 5000, nsub=nsub, drag=drag)
        b = run("warp", prec, 5000, nsub=nsub, drag=drag)
        for p, q in zip(a, b):
            assert np.array_equal(p, q)


def test_ring_atomic_source_fp64():
    a = run("ring", "fp64", 40000, deposit="atomic")
    b = run("warp", "fp64", 40000, deposit="atomic")
    for p, q in zip(a[:3], b[:3]):
        assert np.array_equal(p, q)
    assert np.abs(a[3] - b[3]).max() <= 1e-12 * np.abs(b[3]).max()


def test_ring_matches_oracle_many_tiles():
    """Several tiles per block, a ragged end and a re-sort, against the CPU oracle."""
    npcl, steps = 148 * 1280 * 3 + 333, 3
    xyz, uvw, d = workload.parcels(npcl, 9)
    U = workload.tgv_field(N, dtype=np.float32)
    fs = [workload.fluid_scale(k) for k in range(steps)]
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=2)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(steps):
            h.step(workload.DT, fs[k])
        h.synchronize()
        gx, gu, _ = h.get_parcels()
        gc, gs = h.get_cells(), h.get_source()
    cfg = oracle.make_cfg(N, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=1)
    r = oracle.run(cfg, xyz, uvw, d, U.astype(np.float64), steps, workload.DT, fscale=fs,
                   nthreads=8)
    assert r["status"] == 0
    assert np.array_equal(gx, r["xyz"])
    assert np.array_equal(gu, r["uvw"])
    assert np.array_equal(gc, r["cells"])
    assert np.array_equal(gs, r["src_quant"])


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_overlapped_finalize_same_results(prec):
    """The source conversion of a step on the library's second stream, beside the next step
    (default for one cloud), gives the same parcels and sources on every step as the
    conversion in stream order; a graph captured after overlapped steps replays the same."""
    npcl, steps = 50000, 7
    xyz, uvw, d = workload.parcels(npcl, 13)
    U = workload.tgv_field(N, U0=2.0, dtype=np.float64 if prec == "fp64" else np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision=prec, n_substeps=1,
                    sort_interval=2)
    out = {}
    for on in (True, False):
        with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
            h.set_finalize_overlap(on)
            h.set_parcels(xyz, uvw, d)
            h.set_fluid_velocity(U)
            srcs = []
            for k in range(steps):
                h.step(workload.DT, workload.fluid_scale(k))
                if k % 3 == 2:
                    srcs.append(h.get_source())
            for k in range(3):          # several steps in flight before the next read
                h.step(workload.DT, workload.fluid_scale(steps + k))
            srcs.append(h.get_source())
            h.graph_capture(4, workload.DT)
            h.graph_launch()
            h.synchronize()
            srcs.append(h.get_source())
            x, u, _ = h.get_parcels()
            out[on] = (srcs, x, u, h.get_cells())
    a, b = out[True], out[False]
    for s1, s2 in zip(a[0], b[0]):
        assert np.array_equal(s1, s2)
    for p, q in zip(a[1:], b[1:]):
        assert np.array_equal(p, q)


@pytest.mark.parametrize("prec,nsub", [("mixed", 1), ("fp64", 1), ("mixed", 3)])
def test_tet_ring_equals_warp_kernel(prec, nsub):
    """The tet step on the shared-memory ring (default for one cloud) and on per-warp tiles:
    parcels, owning tets, sources and walk-length histograms identical."""
    n, npcl, steps = 12, 148 * 1024 + 333, 3
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, workload.L_BOX, 0.15, 1)
    xyz, _, d = workload.parcels(npcl, 17)
    uvw = np.random.default_rng(18).normal(0.0, 5.0, (3, npcl)).astype(np.float32).astype(np.float64)
    hint = workload.tet_hints(xyz, hex_ijk, n)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=3.0)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision=prec, n_substeps=nsub,
                    sort_interval=2)
    out = {}
    for kind in ("ring", "warp"):
        with st.ParcelTracker(prm, st.tet_mesh_desc(verts, tets, nbr, 0.0, workload.L_BOX)) as h:
            h.set_step_kernel(kind)
            h.set_parcels(xyz, uvw, d, hint=hint)
            h.set_fluid_velocity(U.astype(np.float64 if prec == "fp64" else np.float32))
            lost = 0
            for k in range(steps):
                h.step(1e-3, workload.fluid_scale(k))
                try:   # fast parcels can outrun the walk's hop limit; both kernels count them
                    h.synchronize()
                except st.ScaleTrackError as e:
                    assert e.code == st.ST_ERR_PARCEL_OUTSIDE, str(e)
                    lost += int(str(e).split(":", 1)[1].split()[0])
            x, u, _ = h.get_parcels()
            out[kind] = (x, u, h.get_cells(), h.get_source(), h.hop_histogram(), lost)
    for p, q in zip(out["ring"], out["warp"]):
        assert np.array_equal(p, q)
    assert out["ring"][4][1:].sum() > 0    # the walks did hop


@pytest.mark.parametrize("kind", ["ring", "warp"])
def test_dense_cells_against_oracle(kind):
    """4^3 cells and 2e5 parcels (about 3000 per cell): after each re-sort nearly every warp
    holds a single cell, so the deposit takes its full-warp reduction; parcels, cells and the
    fixed-point source stay bit-exact with the CPU oracle."""
    n, npcl, steps = 4, 200_000, 3
    xyz, uvw, d = workload.parcels(npcl, 21)
    U = workload.tgv_field(n, dtype=np.float32)
    fs = [workload.fluid_scale(k) for k in range(steps)]
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=1)
    with st.ParcelTracker(prm, st.mesh_desc(n, 0.0, workload.L_BOX)) as h:
        h.set_step_kernel(kind)
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(steps):
            h.step(workload.DT, fs[k])
        h.synchronize()
        gx, gu, _ = h.get_parcels()
        gc, gs = h.get_cells(), h.get_source()
    cfg = oracle.make_cfg(n, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=1)
    r = oracle.run(cfg, xyz, uvw, d, U.astype(np.float64), steps, workload.DT, fscale=fs,
                   nthreads=8)
    assert r["status"] == 0
    assert np.array_equal(gx, r["xyz"])
    assert np.array_equal(gu, r["uvw"])
    assert np.array_equal(gc, r["cells"])
    assert np.array_equal(gs, r["src_quant"])


def test_bounded_wait_reports_fault_and_recovers():
    """Failure detection without a fault: in the stall test every ring block's consumers wait
    on a barrier that nothing completes; after the limit (2e6 cycles, about 1 ms) they record
    it, the producer's wait for them runs out too, the block drains its copies in flight, and
    the host gets an error status instead of a hang.  The device stays usable: with the
    default limit the same handle, given the parcels again, steps to the same results as a
    fresh handle."""
    npcl = 148 * 1280 * 2 + 100
    xyz, uvw, d = workload.parcels(npcl, 23)
    U = workload.tgv_field(N, dtype=np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=0)
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.step(workload.DT, 1.0)            # scale set-up and one normal step
        h.synchronize()
        h.set_wait_limit(2_000_000, stall=True)
        h.step(workload.DT, 1.0)
        with pytest.raises(st.ScaleTrackError) as e:
            h.synchronize()
        assert e.value.code == st.ST_ERR_CUDA and "gave up waiting" in str(e.value)
        assert "fault bits 3" in str(e.value)      # consumers (2) and producer (1)
        h.set_wait_limit(0)
        h.set_parcels(xyz, uvw, d)
        for k in range(2):
            h.step(workload.DT, 1.0)
        h.synchronize()
        a = (*h.get_parcels()[:2], h.get_cells(), h.get_source())
    with st.ParcelTracker(prm, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        for k in range(2):
            h.step(workload.DT, 1.0)
        h.synchronize()
        b = (*h.get_parcels()[:2], h.get_cells(), h.get_source())
    for p, q in zip(a, b):
        assert np.array_equal(p, q)
