"""Benchmark of the B200 Lagrangian parcel step (one JSON line on stdout, rank 0).

Workload: 128^3 uniform hex mesh (2,097,152 cells) on
[0, 0.1 m]^3, 1e7 parcels, Schiller-Naumann drag with explicit Euler, dt = 1e-4 s, one
substep, mixed precision (FP64 positions, FP32 drag/velocity, deterministic fixed-point
source reduced to FP64), Morton re-sort every 20 steps, time-varying Taylor-Green-like
fluid field, seeded synthetic inputs.  A step = one call of the parcel step over every
parcel (including the source finalize and, every 20th step, the re-sort).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

  value      particle-steps/s of the mixed deterministic step, inputs resident in HBM
  e2e        same metric through the reference-facing C ABI (st_evolve_cloud) with pinned
             host exchange arrays: U copied in and the source copied out every step
  roofline   the step kernel's algorithmic bytes / its event-timed duration vs measured HBM
  cpu_baseline  the CPU oracle (restatement of the reference's CPU path) on this host
  fp64_*     the all-FP64 GPU step (same kernel design, FP64 atomics, re-sorted) on the
             same inputs
  fp64_plain_*  the reference's plain method in FP64 on the GPU: parcels in their given
             order, never re-sorted, three FP64 atomics per parcel
--impl reference times the CPU restatement of the reference's path with all host threads.
Multi-GPU (torchrun): every rank steps its own 1e7 parcels (weak scaling) against the
replicated U; the ranks sum their int64 fixed-point accumulators with an NCCL all-reduce and
agree on one scale (the sharded step, st_shard_*), so the source is exact.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "scale-track_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

import workload  # noqa: E402

METRIC = "particle-steps/s mixed vs FP64 on 1 B200 at src rel err<=1e-5; adjoint/fwd cost"
UNIT = "particle-steps/s"
CONFIG = workload.CONFIGS["hex128_mixed"]
FALLBACK_HBM_GBS = 6650.0


def bench_config(npcl, ncells, ws):
    """The workload both arms name in their JSON line (the reference arm steps a bounded
    sample of it on the host cores and says so in cpu_baseline.sample)."""
    return {"workload": "128^3 hex (2,097,152 cells), 1e7 parcels per GPU, Schiller-Naumann "
                        "explicit, dt=1e-4 s, 1 substep, mixed precision, Morton re-sort every "
                        "20 steps, time-varying field",
            "nparcels_per_gpu": npcl, "ncells": ncells, "sort_interval": CONFIG["sort_interval"],
            "l2": "inputs larger than L2: parcel state %d MB per GPU" % (npcl * 40 // 10**6),
            "parallelism": "dp%d (parcels sharded, U replicated, source summed exactly)" % ws}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nparcels", type=int, default=CONFIG["nparcels"])
    ap.add_argument("--ncells", type=int, default=CONFIG["n"], help="cells per direction")
    ap.add_argument("--fp64-steps", type=int, default=100)
    ap.add_argument("--e2e-steps", type=int, default=50)
    ap.add_argument("--accuracy-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-extras", action="store_true", help="only the headline timing")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the configuration-4 adjoint timing")
    ap.add_argument("--no-tets", dest="tets", action="store_false",
                    help="skip the 96^3 x 6 jittered tet mesh workload")
    ap.add_argument("--tet-steps", type=int, default=workload.CONFIGS["tets96x6_mixed"]["steps"])
    ap.add_argument("--tet-nparcels", type=int, default=workload.CONFIGS["tets96x6_mixed"]["nparcels"])
    ap.add_argument("--tets-only", action="store_true",
                    help="time the tet mesh workload alone and print its object (profiling runs)")
    ap.add_argument("--no-clouds", dest="clouds", action="store_false",
                    help="skip the configuration-3 multi-cloud timing")
    ap.add_argument("--clouds-only", action="store_true",
                    help="time the 64-cloud workload alone and print its object (profiling runs)")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="with --clouds-only: skip the autotuner (profiling runs)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ----------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        self.gpu = ids[local_index] if local_index < len(ids) else str(local_index)
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, t0=None, t1=None):
        """Median SM clock and active throttle reasons of the samples taken in [t0, t1]
        (wall-clock seconds); the nearest samples when the region is shorter than the
        200 ms sampling period."""
        if not self.path or not os.path.exists(self.path):
            return None
        import datetime
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 10:
                    continue
                try:
                    ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                except ValueError:
                    continue
                rows.append((ts, parts[1:]))
        os.unlink(self.path)
        if not rows:
            return None
        window = "timed region"
        sel = rows
        if t0 is not None and t1 is not None:
            sel = [r for r in rows if t0 - 0.1 <= r[0] <= t1 + 0.1]
            if not sel:
                mid = 0.5 * (t0 + t1)
                sel = sorted(rows, key=lambda r: abs(r[0] - mid))[:2]
                window = "nearest samples (region shorter than the sampling period)"
        sm = [float(r[1][1]) for r in sel if r[1][1].replace(".", "").isdigit()]
        smax = [float(r[1][2]) for r in sel if r[1][2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, r in sel for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(sel), "window": window}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_parcel(precision):
    """DRAM bytes per parcel of the step kernel from a committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "k_step_traffic.json")
    try:
        with open(p) as f:
            return float(json.load(f)[precision]["dram_bytes_per_parcel"])
    except Exception:
        return None


def ncu_tet_traffic():
    """DRAM bytes per launch of the tet step kernel from a committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "k_step_traffic.json")
    try:
        with open(p) as f:
            return float(json.load(f)["tets"]["dram_bytes_per_launch"])
    except Exception:
        return None


def ncu_instructions_per_parcel_substep(workload_name):
    """Warp instructions per parcel and substep of a step kernel, from a committed ncu
    summary (profiles/instructions.json), or None."""
    p = os.path.join(ROOT, "profiles", "instructions.json")
    try:
        with open(p) as f:
            return json.load(f)[workload_name]
    except Exception:
        return None


def make_params(st, precision, deposit="deterministic", sort_interval=None):
    return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                     drag_model="schiller_naumann", precision=precision, n_substeps=1,
                     deposit=deposit,
                     sort_interval=CONFIG["sort_interval"] if sort_interval is None
                     else sort_interval)


class DeviceTimer:
    """CUDA events recorded on the library's stream (the launching stream)."""

    def __init__(self, torch, stream_ptr, device):
        self.torch = torch
        # the library's own stream, or torch's default stream (pointer 0) when the library
        # was set to run on it (the multi-rank path)
        self.stream = (torch.cuda.ExternalStream(stream_ptr, device=device) if stream_ptr
                       else torch.cuda.default_stream(device))
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)

    def start(self):
        self.a.record(self.stream)

    def stop(self):
        self.b.record(self.stream)
        self.b.synchronize()
        return self.a.elapsed_time(self.b)  # ms


class DevArray:
    """Zero-copy view of a library-owned device array for torch (__cuda_array_interface__)."""

    def __init__(self, ptr, n, typestr="<f8"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


# ----------------------------------------------------------------------------- our arm
def sharded_step(st, torch, h, pg, dev, total):
    """The step of one rank's shard of a cloud of `total` parcels over the process group `pg`
    (torch.distributed): the library runs on torch's current stream, where the collectives
    run; the ranks agree on one fixed-point scale (max of their largest-deposit exponents)
    and sum their int64 accumulators exactly, so every rank converts the same integers and
    the source equals that of one GPU stepping every parcel."""
    st.lib().st_set_stream(h.handle, torch.cuda.current_stream(dev).cuda_stream)
    h.shard_set_total(total)
    acc_p, nacc, exp_p, nexp = h.shard_buffers()
    acc_v = torch.as_tensor(DevArray(acc_p, nacc, "<i8"), device=dev)
    exp_v = torch.as_tensor(DevArray(exp_p, nexp, "<i4"), device=dev)

    def step(dt_, fs_):
        if h.shard_needs_probe(dt_):
            h.shard_probe(dt_, fs_)
            pg.all_reduce(exp_v, op=pg.ReduceOp.MAX)
        h.shard_deposit(dt_, fs_)
        pg.all_reduce(acc_v)
        pg.all_reduce(exp_v, op=pg.ReduceOp.MAX)
        h.shard_finish()
    return step


def run_ours(args):
    import torch
    import scaletrack as st

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    n = args.ncells
    npcl = args.nparcels
    ncells = n ** 3
    xyz, uvw, d = workload.parcels(npcl, CONFIG["seed"] + rank)
    U = workload.tgv_field(n, dtype=np.float32)
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)
    dt = workload.DT
    fs = lambda k: workload.fluid_scale(k, dt, CONFIG["time_varying"])  # noqa: E731

    def barrier_sync():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    extras = {}
    # ---- accuracy: mixed vs all-FP64 on the same inputs ----
    # single-GPU extras run on one rank only when the job has one rank: with several ranks
    # the others would wait in a collective for minutes
    solo = ws == 1
    if not args.no_extras and solo:
        extras.update(accuracy(st, xyz, uvw, d, U, mesh, local, args.accuracy_steps, dt, fs))

    # ---- headline: mixed deterministic step, device-resident ----
    h = st.ParcelTracker(make_params(st, "mixed"), mesh, device=local)
    h.set_parcels(xyz, uvw, d)
    h.set_fluid_velocity(U)
    step = h.step
    if pg is not None:
        step = sharded_step(st, torch, h, pg, dev, ws * npcl)
    timer = DeviceTimer(torch, h.stream(), dev)
    k = 0
    # the clock sampler starts before the warm-up: nvidia-smi's start-up must not overlap
    # the timed region
    clk = ClockSampler(local).__enter__()
    time.sleep(1.5)
    for _ in range(args.warmup):
        step(dt, fs(k))
        k += 1
    h.synchronize()
    barrier_sync()
    launches0 = h.launch_count()
    w0 = time.time()
    timer.start()
    for _ in range(args.steps):
        step(dt, fs(k))
        k += 1
    # the last step's source conversion runs beside the stream: order the stream after it so
    # that the stop event covers it
    h.source_device_ptr(0)
    ms = timer.stop()
    w1 = time.time()
    time.sleep(0.3)
    clk.__exit__(None, None, None)
    launches = h.launch_count() - launches0
    h.synchronize()
    barrier_sync()
    # per-kernel times from the same number of further steps with events around every kernel
    # (outside the timed region: the events perturb it)
    h.profile(True)
    for kind in ("step", "finalize", "sort"):
        h.profile_read(kind, reset=True)
    for _ in range(args.steps):
        step(dt, fs(k))
        k += 1
    nstep, step_ms = h.profile_read("step")
    nfin, fin_ms = h.profile_read("finalize")
    nsort, sort_ms = h.profile_read("sort")
    h.profile(False)
    h.synchronize()
    barrier_sync()
    if pg is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.summary(w0, w1)
    ms_per_step = ms / args.steps
    value = ws * npcl * args.steps / (ms / 1e3)

    peak, peak_src = measured_hbm_peak()
    algo_step = workload.step_kernel_bytes("mixed", npcl, ncells)
    step_avg_ms = step_ms / max(nstep, 1)
    achieved = algo_step / (step_avg_ms / 1e3) / 1e9
    tpp = ncu_traffic_per_parcel("mixed")
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": None if tpp is None else round(tpp * npcl),
                "kernel": "k_step_ring<double,float,DET1,1 substep>", "peak_source": peak_src,
                "algorithmic_bytes_per_launch": algo_step,
                "avg_launch_ms": round(step_avg_ms, 5)}
    whole_step_frac = workload.algorithmic_bytes("mixed", npcl, ncells) / (ms_per_step / 1e3) \
        / 1e9 / peak
    extras["kernel_ms_per_step"] = {"step": round(step_avg_ms, 5),
                                    "finalize": round(fin_ms / max(nfin, 1), 5),
                                    "sort_per_call": round(sort_ms / max(nsort, 1), 5),
                                    "sort_calls": nsort}
    extras["whole_step_hbm_frac"] = round(whole_step_frac, 4)
    h.close()

    # ---- all-FP64 GPU steps on the same inputs: the same kernel design with FP64 atomics
    # (re-sorted like the mixed step), and the reference's plain method in FP64 (one pass
    # over the parcels in their given order, three FP64 atomics per parcel, no re-sort) ----
    def time_fp64(sort_interval):
        with st.ParcelTracker(make_params(st, "fp64", "atomic", sort_interval), mesh,
                              device=local) as h64:
            h64.set_parcels(xyz, uvw, d)
            h64.set_fluid_velocity(U.astype(np.float64))
            t64 = DeviceTimer(torch, h64.stream(), dev)
            for j in range(args.warmup):
                h64.step(dt, fs(j))
            h64.synchronize()
            t64.start()
            for j in range(args.fp64_steps):
                h64.step(dt, fs(args.warmup + j))
            return t64.stop()

    if not args.no_extras and solo and args.fp64_steps > 0:
        ms64 = time_fp64(None)
        extras["fp64_value"] = npcl * args.fp64_steps / (ms64 / 1e3)
        extras["fp64_ms_per_step"] = ms64 / args.fp64_steps
        extras["mixed_over_fp64"] = round(value / ws / extras["fp64_value"], 3)
        ms64p = time_fp64(0)
        extras["fp64_plain_value"] = npcl * args.fp64_steps / (ms64p / 1e3)
        extras["fp64_plain_ms_per_step"] = ms64p / args.fp64_steps
        extras["mixed_over_fp64_plain"] = round(value / ws / extras["fp64_plain_value"], 3)

    # ---- end to end through the reference-facing shim (pinned host exchange arrays) ----
    e2e = None
    if not args.no_extras and args.e2e_steps > 0:
        # every rank drives its own shard through its own default handle; the job's time is
        # the slowest rank's
        st.setup(make_params(st, "mixed"), mesh)
        hd = st.default_handle()
        if st.lib().st_set_parcels(hd, 0, npcl, xyz.ctypes.data, uvw.ctypes.data,
                                   d.ctypes.data) != 0:
            raise RuntimeError(st.last_error())
        Uh = st.allocate_array("U", ncells, 3, 4)
        UT = st.allocate_array("UTrans", ncells, 3, 4)
        Uh[:] = U
        for j in range(args.warmup):
            st.evolve_cloud(dt)
        barrier_sync()
        t0 = time.perf_counter()
        for j in range(args.e2e_steps):
            st.evolve_cloud(dt)
        el = time.perf_counter() - t0
        if pg is not None:
            t = torch.tensor([el], device=dev, dtype=torch.float64)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            el = float(t.item())
        if not np.isfinite(UT).all():
            raise RuntimeError("non-finite source from the coupling shim")
        st.finalize()
        e2e = {"value": ws * npcl * args.e2e_steps / el, "unit": UNIT,
               "h2d_bytes_per_step": ncells * 3 * 4, "d2h_bytes_per_step": ncells * 3 * 4,
               "steps": args.e2e_steps,
               "path": "st_evolve_cloud: U (float32 [nCells][3], pinned) H2D, step, source "
                       "(float32 UTrans, pinned) D2H; fixed fluid scale"}
    if not args.no_extras and args.e2e_steps > 0 and solo:
        # zero-copy exchange: the library's kernels read U from and write UTrans to the
        # pinned pages directly
        st.setup(make_params(st, "mixed"), mesh)
        hd = st.default_handle()
        if st.lib().st_set_parcels(hd, 0, npcl, xyz.ctypes.data, uvw.ctypes.data,
                                   d.ctypes.data) != 0:
            raise RuntimeError(st.last_error())
        Uh = st.allocate_array("U", ncells, 3, 4)
        UT = st.allocate_array("UTrans", ncells, 3, 4)
        Uh[:] = U
        st.set_exchange_mode("mapped")
        for j in range(args.warmup):
            st.evolve_cloud(dt)
        t0 = time.perf_counter()
        for j in range(args.e2e_steps):
            st.evolve_cloud(dt)
        el = time.perf_counter() - t0
        if not np.isfinite(UT).all():
            raise RuntimeError("non-finite source from the coupling shim")
        st.finalize()
        extras["e2e_mapped"] = {
            "value": npcl * args.e2e_steps / el, "unit": UNIT,
            "h2d_bytes_per_step": ncells * 3 * 4, "d2h_bytes_per_step": ncells * 3 * 4,
            "steps": args.e2e_steps,
            "path": "st_evolve_cloud with st_set_exchange_mode(mapped): kernels read U from "
                    "and write UTrans to the pinned host pages (no DMA copies)"}
        # the reference's asynchronous coupling: the step overlaps the next call's copies
        st.setup(make_params(st, "mixed"), mesh)
        hd = st.default_handle()
        if st.lib().st_set_parcels(hd, 0, npcl, xyz.ctypes.data, uvw.ctypes.data,
                                   d.ctypes.data) != 0:
            raise RuntimeError(st.last_error())
        Uh = st.allocate_array("U", ncells, 3, 4)
        UT = st.allocate_array("UTrans", ncells, 3, 4)
        Uh[:] = U
        for j in range(args.warmup):
            st.evolve_cloud_async(dt)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for j in range(args.e2e_steps):
            st.evolve_cloud_async(dt)
        el = time.perf_counter() - t0
        if not np.isfinite(UT).all():
            raise RuntimeError("non-finite source from the coupling shim")
        st.finalize()
        extras["e2e_async"] = {
            "value": npcl * args.e2e_steps / el, "unit": UNIT,
            "h2d_bytes_per_step": ncells * 3 * 4, "d2h_bytes_per_step": ncells * 3 * 4,
            "steps": args.e2e_steps,
            "path": "st_evolve_cloud_async (the reference's default coupling): U H2D and the "
                    "extrapolated source D2H on a copy stream, overlapping the previous step"}

    # ---- 64 clouds in one launch, graph replay, autotuned ----
    if not args.no_extras and solo and args.clouds:
        extras["clouds"] = run_clouds(st, torch, local, dev)

    # ---- face walk on the jittered 96^3 x 6 tet mesh ----
    if not args.no_extras and solo and args.tets:
        extras["tets"] = run_tets(st, torch, local, dev, args.tet_steps, args.tet_nparcels)

    # ---- adjoint of the time-averaged source (128^3 hex, 1e6 parcels) ----
    if not args.no_extras and solo and args.adjoint:
        extras["adjoint"] = run_adjoint(st, local)

    # ---- CPU baseline: the oracle on this host's cores (bounded sample) ----
    cpu = None
    if not args.no_extras and solo and args.cpu_seconds > 0:
        cpu = cpu_rate(n, xyz, uvw, d, U, args.cpu_seconds)
        # the reference's own CPU executor is a serial loop (A:818-823): one thread too
        extras["cpu_baseline_1thread"] = cpu_rate(n, xyz, uvw, d, U, args.cpu_seconds / 3,
                                                  threads=1)

    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 positions / f32 drag+velocity "
        "/ int64 fixed-point source -> f64",
        "data": "synthetic (seeded uniform parcels, lognormal diameters, analytic TGV field)",
        "config": bench_config(npcl, ncells, ws),
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
        "gpu_launches": launches,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


def source_errors(Sm, Sd):
    """Source of the mixed step against the FP64 step's source S: max-norm and L2 relative to
    S, and the per-cell relative error over the cells with |S_c| >= 1e-3 max |S|."""
    mx = np.abs(Sd).max()
    err = np.abs(Sm - Sd)
    sel = np.abs(Sd) >= 1e-3 * mx
    rel = err[sel] / np.abs(Sd[sel])
    return {"max_norm": float(err.max() / mx),
            "l2": float(np.linalg.norm(Sm - Sd) / np.linalg.norm(Sd)),
            "per_cell_p99": float(np.percentile(rel, 99)),
            "per_cell_max": float(rel.max()),
            "per_cell_cells": int(sel.sum())}


def accuracy(st, xyz, uvw, d, U, mesh, local, steps, dt, fs):
    """Mixed against all-FP64 at the benchmark's size: (a) `steps` steps of both from the
    same inputs (arithmetic plus trajectory divergence), (b) one step of both from the mixed
    run's state after `steps` steps (the arithmetic alone, on relaxed parcels)."""
    out = {}
    S, state = {}, {}
    for prec in ("mixed", "fp64"):
        with st.ParcelTracker(make_params(st, prec), mesh, device=local) as h:
            h.set_parcels(xyz, uvw, d)
            h.set_fluid_velocity(U.astype(np.float64 if prec == "fp64" else np.float32))
            for k in range(steps):
                h.step(dt, fs(k))
            h.synchronize()
            S[prec] = h.get_source()
            state[prec] = (h.get_parcels(), h.get_cells())
    (pm, _, _), cm = state["mixed"]
    (pd, _, _), cd = state["fp64"]
    e = source_errors(S["mixed"], S["fp64"])
    out["src_rel_err_mixed_vs_fp64"] = e["max_norm"]
    out["src_rel_err_l2_mixed_vs_fp64"] = e["l2"]
    out["pos_rel_err_mixed_vs_fp64"] = float(np.abs(pm - pd).max() / workload.L_BOX)
    out["cells_differing_mixed_vs_fp64"] = int(np.sum(cm != cd))
    out["accuracy_steps"] = steps
    out["src_err_after_steps"] = dict(e, steps=steps, start="same inputs")
    x1, u1, _ = state["mixed"][0]
    S1, c1 = {}, {}
    for prec in ("mixed", "fp64"):
        with st.ParcelTracker(make_params(st, prec), mesh, device=local) as h:
            h.set_parcels(x1, u1, d)
            h.set_fluid_velocity(U.astype(np.float64 if prec == "fp64" else np.float32))
            h.step(dt, fs(steps))
            h.synchronize()
            S1[prec] = h.get_source()
            c1[prec] = h.get_cells()
    out["src_err_one_step"] = dict(source_errors(S1["mixed"], S1["fp64"]),
                                   start="mixed state after %d steps, one step of each" % steps,
                                   cells_differing=int(np.sum(c1["mixed"] != c1["fp64"])))
    return out


def run_clouds(st, torch, local, dev, tune=True):
    """64 clouds with log-uniform sizes on a 64^3 mesh, each with its own
    source, one persistent launch per step; block size and re-sort interval from the
    autotuner; the step sequence replayed from a captured CUDA graph."""
    c = workload.CONFIGS["clouds64_hex64"]
    sizes, dmed = workload.cloud_sizes(c)
    n = c["n"]
    U = workload.tgv_field(n, dtype=np.float32)
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision="mixed",
                    n_substeps=c["substeps"], n_clouds=c["nclouds"], sort_interval=20)
    total = int(sizes.sum())
    with st.ParcelTracker(prm, st.mesh_desc(n, 0.0, workload.L_BOX), local) as h:
        for k in range(c["nclouds"]):
            xyz, uvw, d = workload.parcels(int(sizes[k]), 1000 + k, d_median=float(dmed[k]))
            h.set_parcels(xyz, uvw, d, cloud=k)
        h.set_fluid_velocity(U)
        if tune:
            tune = h.autotune(workload.DT, trial_steps=40)
        else:   # profiling runs: the handle's defaults, no trial launches
            tune = {"block_size": prm.block_size or 256, "sort_interval": prm.sort_interval,
                    "note": "autotuner skipped"}
        si = tune["sort_interval"]
        chunk = 2 * si if si else 20
        timer = DeviceTimer(torch, h.stream(), dev)
        # plain launches
        for _ in range(3):
            h.step(workload.DT)
        h.synchronize()
        steps = (c["steps"] // chunk) * chunk
        h.profile(True)
        h.profile_read("step", reset=True)
        timer.start()
        for _ in range(steps):
            h.step(workload.DT)
        ms_plain = timer.stop()
        nst, st_ms = h.profile_read("step")
        h.profile(False)
        # captured graph (capture right after a re-sort: run up to the next one first)
        h.synchronize()
        extra = (si - (3 + steps) % si) % si if si else 0
        for _ in range(extra):
            h.step(workload.DT)
        h.graph_capture(chunk, workload.DT)
        h.graph_launch()
        h.synchronize()
        timer.start()
        for _ in range(steps // chunk):
            h.graph_launch()
        ms_graph = timer.stop()
        h.synchronize()
    peak, peak_src = measured_hbm_peak()
    step_avg = st_ms / max(nst, 1)
    algo = workload.step_kernel_bytes("mixed", total, n ** 3)
    inst = ncu_instructions_per_parcel_substep("clouds64_hex64")
    roof = {"bound": "issue: ten substeps of the parcel arithmetic per parcel in registers "
                     "for each load and store of its state",
            "kernel": "k_step<double,float,DET1,substeps,clouds> (all 64 clouds, one launch)",
            "algorithmic_bytes_per_launch": algo, "avg_launch_ms": round(step_avg, 5),
            "achieved": round(algo / (step_avg / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
            "peak_source": peak_src,
            "frac": round(algo / (step_avg / 1e3) / 1e9 / peak, 4)}
    if inst is not None:
        # warp instructions issued per second against 4 per SM and clock (148 SMs, 1965 MHz)
        rate = inst["warp_instructions_per_parcel_substep"] * total * c["substeps"] / \
            (step_avg / 1e3)
        roof["issue"] = {"warp_instructions_per_s": rate,
                         "peak_warp_instructions_per_s": 148 * 4 * 1.965e9,
                         "frac": round(rate / (148 * 4 * 1.965e9), 4),
                         "instructions_from": inst["summary"]}
    return {"workload": "64 clouds, sizes log-uniform in [1e3, 2e6] (seed 2), "
                        "median diameter per cloud uniform in [5, 50] um, 64^3 mesh, one "
                        "source per cloud, mixed precision, 10 substeps inside one launch per "
                        "step",
            "parcels": total, "steps": steps, "autotune": tune, "roofline": roof,
            "particle_steps_per_s_graph": total * steps / (ms_graph / 1e3),
            "particle_steps_per_s_launches": total * steps / (ms_plain / 1e3),
            "ms_per_step_graph": ms_graph / steps, "ms_per_step_launches": ms_plain / steps}


def run_tets(st, torch, local, dev, steps, npcl=None):
    """96^3 hexes split into 6 jittered tets (5,308,416 tets), 2e7 parcels,
    carrier field U0 = 3 m/s at the tet centroids, Schiller-Naumann, one substep, mixed
    precision, greedy face walk after every position update, re-sort by owning tet every 10
    steps."""
    c = workload.CONFIGS["tets96x6_mixed"]
    n, dt = c["n"], workload.DT
    npcl = npcl or c["nparcels"]
    verts, tets, nbr, hex_ijk = workload.kuhn_tet_mesh(n, workload.L_BOX, c["jitter"],
                                                       c["mesh_seed"])
    xyz, uvw, d = workload.parcels(npcl, c["seed"])
    hint = workload.tet_hints(xyz, hex_ijk, n)
    U = workload.tgv_at(workload.tet_centroids(verts, tets), U0=c["U0"])
    prm = st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                    drag_model="schiller_naumann", precision=c["precision"], n_substeps=1,
                    sort_interval=c["sort_interval"])
    desc = st.tet_mesh_desc(verts, tets, nbr, 0.0, workload.L_BOX)
    lost = [0]

    def sync(h):
        # A parcel whose walk exceeds the hop limit is held in place and reported; with
        # explicit Euler at dt = 1e-4 s the rare parcels below ~4 um (dt / tau > 2) are
        # numerically unstable and eventually outrun any walk.  The oracle does the same.
        try:
            h.synchronize()
        except st.ScaleTrackError as e:
            if e.code != st.ST_ERR_PARCEL_OUTSIDE:
                raise
            lost[0] += int(str(e).split(":", 1)[1].split()[0])

    with st.ParcelTracker(prm, desc, local) as h:
        h.set_parcels(xyz, uvw, d, hint=hint)
        del xyz, uvw, d, hint
        h.set_fluid_velocity(U)
        k = 0
        for _ in range(5):
            h.step(dt, workload.fluid_scale(k))
            k += 1
        sync(h)
        h.hop_histogram(reset=True)
        h.profile(True)
        for kind in ("step", "sort", "finalize"):
            h.profile_read(kind, reset=True)
        timer = DeviceTimer(torch, h.stream(), dev)
        timer.start()
        for _ in range(steps):
            h.step(dt, workload.fluid_scale(k))
            k += 1
        ms = timer.stop()
        nstep, step_ms = h.profile_read("step")
        nsort, sort_ms = h.profile_read("sort")
        nfin, fin_ms = h.profile_read("finalize")
        h.profile(False)
        hops = h.hop_histogram()
        sync(h)
    peak, peak_src = measured_hbm_peak()
    step_avg = step_ms / max(nstep, 1)
    algo = workload.tet_step_kernel_bytes(c["precision"], npcl, tets.shape[0])
    walks = float(hops.sum())
    return {"workload": "96^3 x 6 jittered tets (5,308,416), 2e7 parcels, "
                        "U0 = 3 m/s, Schiller-Naumann, dt = 1e-4 s, 1 substep, mixed precision, "
                        "face walk, re-sort by owning tet every %d steps" % c["sort_interval"],
            "parcels": npcl, "tets": int(tets.shape[0]), "steps": steps,
            "particle_steps_per_s": npcl * steps / (ms / 1e3), "ms_per_step": ms / steps,
            "kernel_ms": {"step": round(step_avg, 5),
                          "sort_per_call": round(sort_ms / max(nsort, 1), 5),
                          "finalize": round(fin_ms / max(nfin, 1), 5)},
            "roofline_step": {"bound": "hbm", "algorithmic_bytes_per_launch": algo,
                              "traffic": ncu_tet_traffic(),
                              "achieved": round(algo / (step_avg / 1e3) / 1e9, 1),
                              "peak": peak, "unit": "GB/s", "peak_source": peak_src,
                              "frac": round(algo / (step_avg / 1e3) / 1e9 / peak, 4)},
            "hop_histogram": [int(v) for v in hops],
            "lost_parcel_steps": lost[0],
            "mean_hops_per_walk": float((hops * np.minimum(np.arange(8), 7)).sum() / walks)
            if walks else 0.0}


def run_adjoint(st, device):
    """Forward (objective) and pull-back (gradient) times of the adjoint workload: J = |Sbar -
    S*|^2 over 200 steps, 1e6 parcels, 128^3 cells, checkpoints every 20 steps."""
    c = workload.CONFIGS["adjoint_hex128"]
    n, npcl, T, C = c["n"], c["nparcels"], c["steps"], c["checkpoint"]
    xyz, uvw, d = workload.parcels(npcl, c["seed"])
    U = workload.tgv_field(n, dtype=np.float32)
    mesh = st.mesh_desc(n, 0.0, workload.L_BOX)

    def prm(alpha=1.0, s=1.0):
        return st.params(mu_c=workload.MU_F, rho_c=workload.RHO_F, rho_d=workload.RHO_P,
                         drag_model="schiller_naumann", precision="mixed", n_substeps=1,
                         drag_multiplier=alpha, diameter_scale=s, sort_interval=20)

    with st.ParcelTracker(prm(c["target_alpha"], c["target_dscale"]), mesh, device) as ht:
        ht.set_parcels(xyz, uvw, d)
        ht.set_fluid_velocity(U)
        target = ht.mean_source_forward(T, C, workload.DT)
    with st.ParcelTracker(prm(), mesh, device) as h:
        h.set_parcels(xyz, uvw, d)
        h.set_fluid_velocity(U)
        h.mean_source_forward(T, C, workload.DT)  # warm-up
        h.mean_source_pullback(np.zeros((n ** 3, 3)), T, C, workload.DT, want_v0=False)
        h.profile(True)
        h.profile_read("adj_forward", reset=True)
        reps = 3
        for _ in range(reps):
            S = h.mean_source_forward(T, C, workload.DT)
            r = S - target
            J = float(np.sum(r * r))
            da, ds, dv0 = h.mean_source_pullback(2.0 * r, T, C, workload.DT)
        nf, fwd_ms = h.profile_read("adj_forward")
        nb, bwd_ms = h.profile_read("adj_reverse")
        h.profile(False)
    fwd = fwd_ms / reps
    bwd = bwd_ms / reps
    return {"workload": "adjoint, 128^3 hex, 1e6 parcels, 200 steps, checkpoints every "
                        "20 steps, mixed precision, J = |mean source - target|^2, target from "
                        "drag x1.1 and diameters x0.95",
            "forward_ms": round(fwd, 3), "pullback_ms": round(bwd, 3),
            "adjoint_over_forward": round(bwd / fwd, 3),
            "forward_particle_steps_per_s": npcl * T / (fwd / 1e3),
            "objective": J, "dJ_ddrag_multiplier": da, "dJ_ddiameter_scale": ds,
            "dJ_dv0_l2": float(np.linalg.norm(dv0))}


def cpu_rate(n, xyz, uvw, d, U, budget_s, threads=None):
    """The CPU oracle (mixed precision, same physics) on a bounded sample of the workload."""
    import oracle
    threads = threads or len(os.sched_getaffinity(0))
    cfg = oracle.make_cfg(n, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=1)
    U64 = U.astype(np.float64)
    # calibrate on a small sample, then size the measured sample to the time budget
    m = min(200_000, d.size)
    t0 = time.perf_counter()
    oracle.run(cfg, xyz[:, :m], uvw[:, :m], d[:m], U64, 1, workload.DT, want_seq=False,
               nthreads=threads)
    t1 = time.perf_counter() - t0
    rate0 = m / max(t1, 1e-6)
    steps = 3
    m2 = int(min(d.size, max(m, rate0 * budget_s / steps)))
    t0 = time.perf_counter()
    oracle.run(cfg, xyz[:, :m2], uvw[:, :m2], d[:m2], U64, steps, workload.DT,
               fscale=[workload.fluid_scale(k) for k in range(steps)], want_seq=False,
               nthreads=threads)
    el = time.perf_counter() - t0
    return {"value": m2 * steps / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{m2} parcels x {steps} steps of the same 128^3 workload "
                      f"(deterministic fixed-point source), {threads} OpenMP threads"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's path on the host cores: its CPU executor (a serial loop over the
    parcels calling evolve_particle!, asyncParallelTracking.jl:818-823) restated in C++ (the
    oracle; Julia is not available), parallelised over all host threads."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    import oracle
    threads = len(os.sched_getaffinity(0))
    n = args.ncells
    npcl = args.nparcels
    xyz, uvw, d = workload.parcels(npcl, CONFIG["seed"])
    U = workload.tgv_field(n, dtype=np.float32).astype(np.float64)
    cfg = oracle.make_cfg(n, 0.0, workload.L_BOX, workload.MU_F, workload.RHO_F,
                          workload.RHO_P, drag="sn_explicit", precision="mixed", n_substeps=1)
    # bounded per-step sample so that warmup + steps finish in a few minutes
    m = min(100_000, npcl)
    t0 = time.perf_counter()
    oracle.run(cfg, xyz[:, :m], uvw[:, :m], d[:m], U, 1, workload.DT, want_quant=False,
               nthreads=threads)
    per = (time.perf_counter() - t0) / m
    total_steps = args.warmup + args.steps
    budget = 150.0
    sample = int(max(10_000, min(npcl, budget / max(total_steps, 1) / max(per, 1e-9))))
    xs, us, ds = xyz[:, :sample].copy(), uvw[:, :sample].copy(), d[:sample]
    fsw = [workload.fluid_scale(k) for k in range(args.warmup)]
    # the reference's own accumulation: a plain sum into UTrans (A:706), no fixed point
    r = oracle.run(cfg, xs, us, ds, U, args.warmup, workload.DT, fscale=fsw, want_quant=False,
                   nthreads=threads)
    fst = [workload.fluid_scale(args.warmup + k) for k in range(args.steps)]
    t0 = time.perf_counter()
    oracle.run(cfg, r["xyz"], r["uvw"], ds, U, args.steps, workload.DT, fscale=fst,
               want_quant=False, nthreads=threads)
    el = time.perf_counter() - t0
    value = sample * args.steps / el
    desc = (f"{sample} of {npcl} parcels per step (128^3 mesh, same physics and inputs), "
            f"{threads} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 positions / f32 drag+velocity",
        "data": "synthetic (seeded uniform parcels, lognormal diameters, analytic TGV field)",
        "config": bench_config(npcl, n ** 3, ws),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.clouds_only:
        import torch
        import scaletrack as st
        torch.cuda.set_device(0)
        print(json.dumps(run_clouds(st, torch, 0, torch.device("cuda", 0), a.tune)), flush=True)
    elif a.tets_only:
        import torch
        import scaletrack as st
        torch.cuda.set_device(0)
        print(json.dumps(run_tets(st, torch, 0, torch.device("cuda", 0), a.tet_steps,
                                  a.tet_nparcels)), flush=True)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
