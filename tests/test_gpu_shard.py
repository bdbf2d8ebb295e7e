"""GPU test of the sharded step (st_shard_*): one cloud split unevenly over two handles on one
GPU, their exponents max-reduced and their fixed-point accumulators summed between the phases
(what an NCCL all-reduce does across GPUs), must give a source bit-identical to one handle
stepping every parcel -- on every step, across re-sorts, in mixed and FP64 precision.  The
two handles stand for two ranks; their kernels never wait on each other."""
import numpy as np
import pytest

import scaletrack as st
import workload

pytestmark = pytest.mark.gpu

N = 20


class DevArray:
    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def params(prec):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision=prec, n_substeps=1,
                     sort_interval=2)


def views(torch, h):
    acc, nacc, ex, nex = h.shard_buffers()
    return (torch.as_tensor(DevArray(acc, nacc, "<i8"), device="cuda"),
            torch.as_tensor(DevArray(ex, nex, "<i4"), device="cuda"))


def allreduce(torch, hs, with_acc):
    for h in hs:
        h.synchronize()
    v = [views(torch, h) for h in hs]
    e = torch.stack([x[1] for x in v]).amax(dim=0)
    s = sum(x[0] for x in v) if with_acc else None
    for a, ex in v:
        ex.copy_(e)
        if with_acc:
            a.copy_(s)
    torch.cuda.synchronize()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_two_shards_equal_one_handle(prec):
    torch = pytest.importorskip("torch")
    n, steps, cut = 60000, 6, 17000
    xyz, uvw, d = workload.parcels(n, 21)
    U = workload.tgv_field(N, U0=2.0, dtype=np.float64 if prec == "fp64" else np.float32)
    mesh = st.mesh_desc(N, 0.0, workload.L_BOX)
    with st.ParcelTracker(params(prec), mesh) as hc, \
            st.ParcelTracker(params(prec), mesh) as ha, \
            st.ParcelTracker(params(prec), mesh) as hb:
        hc.set_parcels(xyz, uvw, d)
        ha.set_parcels(xyz[:, :cut], uvw[:, :cut], d[:cut])
        hb.set_parcels(xyz[:, cut:], uvw[:, cut:], d[cut:])
        for h in (hc, ha, hb):
            h.set_fluid_velocity(U)
        for h in (ha, hb):
            h.shard_set_total(n)
        for k in range(steps):
            dt, fs = workload.DT, workload.fluid_scale(k)
            hc.step(dt, fs)
            if ha.shard_needs_probe(dt):
                assert hb.shard_needs_probe(dt)
                ha.shard_probe(dt, fs)
                hb.shard_probe(dt, fs)
                allreduce(torch, (ha, hb), with_acc=False)
            ha.shard_deposit(dt, fs)
            hb.shard_deposit(dt, fs)
            allreduce(torch, (ha, hb), with_acc=True)
            ha.shard_finish()
            hb.shard_finish()
            hc.synchronize()
            sc = hc.get_source()
            assert np.abs(sc).max() > 0
            assert np.array_equal(ha.get_source(), sc), k
            assert np.array_equal(hb.get_source(), sc), k
        xa, ua, _ = ha.get_parcels()
        xb, ub, _ = hb.get_parcels()
        xc, uc, _ = hc.get_parcels()
        assert np.array_equal(np.concatenate([xa, xb], axis=1), xc)
        assert np.array_equal(np.concatenate([ua, ub], axis=1), uc)


def test_shard_phases_are_checked():
    with st.ParcelTracker(params("mixed"), st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        xyz, uvw, d = workload.parcels(1000, 3)
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(workload.tgv_field(N, dtype=np.float32))
        with pytest.raises(st.ScaleTrackError):   # the first sharded step needs the probe
            h.shard_deposit(workload.DT)
    atomic = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                       drag_model="schiller_naumann", precision="fp64", deposit="atomic")
    with st.ParcelTracker(atomic, st.mesh_desc(N, 0.0, workload.L_BOX)) as h:
        with pytest.raises(st.ScaleTrackError):   # float atomics have no exact sum
            h.shard_set_total(10)
