"""Multi-rank path on the CPU (gloo, world size 2): parcels sharded over ranks, U replicated.
Each rank steps its shard with the CPU oracle (no GPU here) following the protocol of the
library's sharded step (st_shard_*): the ranks agree on one fixed-point scale (max of their
largest-deposit exponents, headroom for the parcels of all ranks), sum their raw int64
accumulators exactly, and convert once.  The source must then equal, bit for bit and on
every step, the source of one process stepping every parcel; the timing rule (maximum over
ranks) is checked the same way."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
import workload

N, NPCL, STEPS = 12, 6000, 4
EXP_NONE = -100000


def _cfg(prec):
    return oracle.make_cfg(N, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                           workload.RHO_P, drag="sn_explicit", precision=prec, n_substeps=1,
                           quant_limbs=2 if prec == "fp64" else 1, deposit_bound=NPCL)


def _shard(rank, world):
    """uneven split: rank r holds parcels [cut_r, cut_r+1) with cut_r = r * 3N / (2 world)"""
    xyz, uvw, d = workload.parcels(NPCL, 7)
    cuts = [min(NPCL, r * 3 * NPCL // (2 * world)) for r in range(world)] + [NPCL]
    sl = slice(cuts[rank], cuts[rank + 1])
    return xyz[:, sl], uvw[:, sl], d[sl]


def _to_source(acc, L, limbs):
    """int64 accumulators -> FP64 source, as the library's finalize converts them"""
    if limbs == 1:
        v = acc.astype(np.float64)
    else:
        hi = acc[0::2] + (acc[1::2] >> 32)
        lo = acc[1::2] & 0xffffffff
        v = hi.astype(np.float64) * 4294967296.0 + lo.astype(np.float64)
    return np.ldexp(v, L).reshape(-1, 3)


def _worker(rank, world, port, prec, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = _cfg(prec)
        U = workload.tgv_field(N).astype(np.float64)
        xyz, uvw, d = _shard(rank, world)
        fs = [workload.fluid_scale(k) for k in range(STEPS)]
        # probe of the first step: the scale every rank uses
        p = oracle.run(cfg, xyz, uvw, d, U, 0, workload.DT, fscale=fs[:1], want_seq=False)
        e = torch.tensor([p["emax"]], dtype=torch.int64)
        dist.all_reduce(e, op=dist.ReduceOp.MAX)
        H = p["H"]
        L = int(e.item()) - H
        sources = []
        for k in range(STEPS):
            r = oracle.run(cfg, xyz, uvw, d, U, 1, workload.DT, fscale=[fs[k]], want_seq=False,
                           scale=L, want_acc=True)
            assert r["overflow"] == 0
            xyz, uvw = r["xyz"], r["uvw"]
            acc = torch.from_numpy(r["acc"].copy())
            dist.all_reduce(acc)                              # exact: integer sum
            sources.append(_to_source(acc.numpy(), L, cfg.quant_limbs))
            e = torch.tensor([r["emax"]], dtype=torch.int64)
            dist.all_reduce(e, op=dist.ReduceOp.MAX)          # next scale, agreed
            if int(e.item()) != EXP_NONE:
                L = int(e.item()) - H
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)              # device time: max over ranks
        if rank == 0:
            out.put((sources, float(t.item())))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_sharded_source_equals_single_process(prec):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, prec, q)) for r in range(world)]
    for p in procs:
        p.start()
    sources, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cfg = _cfg(prec)
    U = workload.tgv_field(N).astype(np.float64)
    xyz, uvw, d = workload.parcels(NPCL, 7)
    scale = oracle.INT_MIN
    for k in range(STEPS):
        r = oracle.run(cfg, xyz, uvw, d, U, 1, workload.DT, fscale=[workload.fluid_scale(k)],
                       scale=scale)
        xyz, uvw, scale = r["xyz"], r["uvw"], r["scale"]
        assert np.abs(r["src_quant"]).max() > 0
        assert np.array_equal(sources[k], r["src_quant"]), k
        # and the fixed-point source is the FP64 sum to its resolution
        ref = r["src_seq"]
        tol = 1e-8 if prec == "mixed" else 1e-14
        assert np.abs(sources[k] - ref).max() <= tol * np.abs(ref).max()
    assert tmax == 2.0
