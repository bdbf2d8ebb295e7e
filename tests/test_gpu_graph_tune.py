"""GPU tests of the multi-cloud path (64 clouds of log-uniform sizes in the benchmark): one launch for all clouds, CUDA-graph
replay of a step sequence and the autotuner.  Replays must give the same bits as st_step
calls, and tuning must not change results (parcel order never changes a parcel's state or
the fixed-point source)."""
import numpy as np
import pytest

import oracle
import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

N = 16


def clouds(k=5, seed=2):
    cfg = dict(workload.CONFIGS["clouds64_hex64"], nclouds=k, size_min=50, size_max=20000,
               seed=seed)
    sizes, dmed = workload.cloud_sizes(cfg)
    out = []
    for c in range(k):
        xyz, uvw, d = workload.parcels(int(sizes[c]), 100 + c, d_median=dmed[c])
        out.append((xyz, uvw, d))
    return out


def params(k, sort_interval=0, nsub=10):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision="mixed", n_substeps=nsub,
                     n_clouds=k, sort_interval=sort_interval)


def run(k, cl, U, steps, graph=False, sort_interval=0, tune=False):
    with st.ParcelTracker(params(k, sort_interval), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        for c, (xyz, uvw, d) in enumerate(cl):
            h.set_parcels(xyz, uvw, d, cloud=c)
        h.set_fluid_velocity(U)
        if tune:
            r = h.autotune(workload.DT, trial_steps=40)
            assert r["block_size"] in (128, 256) and r["sort_interval"] in (0, 10, 20, 40)
            assert r["ms_per_step"] > 0
        if graph:
            chunk = 2 * sort_interval if sort_interval else steps
            h.graph_capture(chunk, workload.DT)
            for _ in range(steps // chunk):
                h.graph_launch()
        else:
            for _ in range(steps):
                h.step(workload.DT)
        h.synchronize()
        return [(h.get_parcels(c)[0], h.get_cells(c), h.get_source(c)) for c in range(k)]


def test_graph_replay_equals_steps():
    cl = clouds()
    U = workload.tgv_field(N, dtype=np.float32)
    a = run(5, cl, U, 12)
    b = run(5, cl, U, 12, graph=True)
    c = run(5, cl, U, 12, graph=True, sort_interval=3)
    for x, y, z in zip(a, b, c):
        for p, q, r in zip(x, y, z):
            assert np.array_equal(p, q) and np.array_equal(p, r)


def test_multi_cloud_against_oracle_per_cloud():
    cl = clouds(6, seed=4)
    U = workload.tgv_field(N, dtype=np.float32)
    g = run(6, cl, U, 4, graph=True)
    cfg = oracle.make_cfg(N, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=10)
    for c, (xyz, uvw, d) in enumerate(cl):
        r = oracle.run(cfg, xyz, uvw, d, U.astype(np.float64), 4, workload.DT)
        assert np.array_equal(g[c][0], r["xyz"])
        assert np.array_equal(g[c][1], r["cells"])
        assert np.array_equal(g[c][2], r["src_quant"])


def test_autotune_does_not_change_results():
    cl = clouds(4, seed=7)
    U = workload.tgv_field(N, dtype=np.float32)
    a = run(4, cl, U, 10)
    b = run(4, cl, U, 10, tune=True)
    for x, y in zip(a, b):
        for p, q in zip(x, y):
            assert np.array_equal(p, q)
