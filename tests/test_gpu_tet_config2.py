"""The face-walk workload at its configured size, checked at every step: 96^3 hexes split
into 6 jittered tets (5,308,416 tets), 2e7 parcels, U0 = 3 m/s, mixed precision, re-sort by
owning tet every 10 steps, 40 steps.  Before and after every step a fixed sample of parcels
-- 1e5 drawn at random plus the 200 with the smallest diameters, where explicit Euler at
dt = 1e-4 s goes unstable and walks can exceed the hop limit -- is read back from the GPU
(st_get_parcel_sample), and the CPU oracle steps the sample's start state (start tet,
position, velocity): owning tets, positions and velocities after the step must be identical,
and so must the lost parcels.  Every parcel the GPU reports lost over the run must be one the
oracle loses in the sample (the relocation rule of A:1303-1335 applied on the tet mesh)."""
import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

L = workload.L_BOX
STEPS = 40
SAMPLE = 100_000


def test_tet_workload_every_step_against_cpu_walk():
    cfg = workload.CONFIGS["tets96x6_mixed"]
    n, npcl = cfg["n"], cfg["nparcels"]
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, L, cfg["jitter"], cfg["mesh_seed"])
    xyz, uvw, d = workload.parcels(npcl, cfg["seed"])
    hint = workload.tet_hints(xyz, hex_ijk, n)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=cfg["U0"])
    rng = np.random.default_rng(77)
    ids = np.union1d(rng.choice(npcl, SAMPLE, replace=False),
                     np.argsort(d, kind="stable")[:200]).astype(np.int32)
    ds = d[ids].copy()
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                    sort_interval=cfg["sort_interval"])
    ocfg = oracle.make_cfg(1, 0.0, L, workload.MU_F, workload.RHO_F, workload.RHO_P,
                           drag="sn_explicit", precision="mixed", n_substeps=1)
    U64 = U.astype(np.float32).astype(np.float64)
    mesh = (verts, tets, nbr)
    lost_gpu = lost_cpu = 0
    with st.ParcelTracker(prm, st.tet_mesh_desc(verts, tets, nbr, 0.0, L)) as h:
        h.set_parcels(xyz, uvw, d, hint=hint)
        del xyz, uvw, hint
        h.set_fluid_velocity(U.astype(np.float32))
        x0, u0, c0 = h.get_parcel_sample(ids)
        for k in range(STEPS):
            fs = workload.fluid_scale(k)
            h.step(workload.DT, fs)
            try:
                h.synchronize()
            except st.ScaleTrackError as e:   # lost parcels of this step, over the cloud
                assert e.code == st.ST_ERR_PARCEL_OUTSIDE, str(e)
                lost_gpu += int(str(e).split(":", 1)[1].split()[0])
            x1, u1, c1 = h.get_parcel_sample(ids)
            r = oracle.tet_run(ocfg, mesh, x0, u0, ds, c0, U64, 1, workload.DT, fscale=[fs],
                               want_seq=False, want_quant=False)
            assert np.array_equal(c1, r["cells"]), k
            assert np.array_equal(x1, r["xyz"]), k
            assert np.array_equal(u1, r["uvw"]), k
            lost_cpu += r["lost"]
            x0, u0, c0 = x1, u1, c1
    assert lost_gpu == lost_cpu, (lost_gpu, lost_cpu)
