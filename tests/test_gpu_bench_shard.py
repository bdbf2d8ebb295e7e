"""GPU test of the benchmark's multi-GPU step (`bench.sharded_step`) on a one-rank NCCL
process group.  The step runs the shard protocol (common scale from the max-reduced
exponents, int64 accumulators summed by `all_reduce`, one conversion) through
torch.distributed on torch's current stream, the way every rank of a multi-GPU run does.
With one rank the collectives are identities, so the parcels and the source must be
bit-identical to the plain step of a handle holding the same parcels, on every step and
across re-sorts.  One rank only: no kernel waits on another GPU."""
import importlib.util
import os
import socket

import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("st_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_bench_sharded_step_on_one_rank_equals_plain_step(prec):
    torch = pytest.importorskip("torch")
    import datetime

    import torch.distributed as dist

    bench = _bench()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, ncell, steps = 50000, 24, 8
    xyz, uvw, d = workload.parcels(n, 31)
    U = workload.tgv_field(ncell, U0=2.0, dtype=np.float64 if prec == "fp64" else np.float32)
    mesh = st.mesh_desc(ncell, 0.0, workload.L_BOX)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision=prec, n_substeps=1,
                    sort_interval=3)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=dev)
    try:
        with st.ParcelTracker(prm, mesh) as hc, st.ParcelTracker(prm, mesh) as hs:
            for h in (hc, hs):
                h.set_parcels(xyz, uvw, d)
                h.set_fluid_velocity(U)
            step = bench.sharded_step(st, torch, hs, dist, dev, n)
            for k in range(steps):
                fs = workload.fluid_scale(k)
                hc.step(workload.DT, fs)
                step(workload.DT, fs)
                hc.synchronize()
                hs.synchronize()
                sc, ss = hc.get_source(), hs.get_source()
                assert np.abs(sc).max() > 0
                assert np.array_equal(sc, ss), f"source differs at step {k + 1}"
            xc, uc, _ = hc.get_parcels()
            xs, us, _ = hs.get_parcels()
            assert np.array_equal(xc, xs) and np.array_equal(uc, us)
            # the rest of a rank's timed loop: CUDA events on the stream the library now
            # shares with torch, the stop after the last source, the slowest rank's time
            timer = bench.DeviceTimer(torch, hs.stream(), dev)
            torch.cuda.synchronize()
            dist.barrier()
            timer.start()
            for k in range(3):
                step(workload.DT, workload.fluid_scale(steps + k))
            hs.source_device_ptr(0)
            ms = timer.stop()
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            assert float(t.item()) == ms > 0.0
    finally:
        dist.destroy_process_group()
