"""Multi-rank path on the CPU (gloo, world size 2): parcels sharded over ranks, U replicated,
the per-cell source summed over ranks.  Each rank steps its shard with the CPU oracle (no
GPU here) and the all-reduced source must equal the source of one process stepping every
parcel; the timing rule (maximum over ranks) is checked the same way."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
import workload

N, NPCL, STEPS = 12, 6000, 3


def _cfg():
    return oracle.make_cfg(N, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                           workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=1)


def _shard(rank, world):
    xyz, uvw, d = workload.parcels(NPCL, 7)
    sl = slice(rank * NPCL // world, (rank + 1) * NPCL // world)
    return xyz[:, sl], uvw[:, sl], d[sl]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        U = workload.tgv_field(N).astype(np.float64)
        xyz, uvw, d = _shard(rank, world)
        fs = [workload.fluid_scale(k) for k in range(STEPS)]
        r = oracle.run(_cfg(), xyz, uvw, d, U, STEPS, workload.DT, fscale=fs, want_quant=False)
        src = torch.from_numpy(r["src_seq"].copy())
        dist.all_reduce(src)                                 # the source exchange
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)             # device time: max over ranks
        if rank == 0:
            out.put((src.numpy(), float(t.item())))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_sharded_source_equals_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world = 2
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    src, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    U = workload.tgv_field(N).astype(np.float64)
    xyz, uvw, d = workload.parcels(NPCL, 7)
    fs = [workload.fluid_scale(k) for k in range(STEPS)]
    ref = oracle.run(_cfg(), xyz, uvw, d, U, STEPS, workload.DT, fscale=fs, want_quant=False)
    ref_src = ref["src_seq"]
    assert np.abs(src - ref_src).max() <= 1e-12 * np.abs(ref_src).max()
    assert tmax == 2.0
