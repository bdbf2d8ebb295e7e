"""CPU checks of the benchmark's host-side figures: the mixed-vs-FP64 source error norms and
the algorithmic-byte model that the roofline divides by (the per-parcel and per-cell bytes of
the step: mixed 76 + 36, FP64 104 + 48, tets 84 + 156)."""
import importlib.util
import os

import numpy as np

import workload

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("st_bench_host", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_source_error_norms():
    bench = _bench()
    S = np.array([[1.0, -2.0, 0.5], [4.0, 1e-4, -1e-5]])
    Sm = S.copy()
    Sm[0, 1] += 2e-6          # relative 1e-6 in a large cell
    Sm[1, 1] += 1e-8          # relative 1e-4 in a cell at 2.5e-5 of the largest: not counted
    e = bench.source_errors(Sm, S)
    assert np.isclose(e["max_norm"], 2e-6 / 4.0)
    assert np.isclose(e["l2"], np.linalg.norm(Sm - S) / np.linalg.norm(S))
    assert e["per_cell_cells"] == 4          # |S| >= 1e-3 * 4 keeps 1, 2, 0.5 and 4
    assert np.isclose(e["per_cell_max"], 1e-6)
    assert e["per_cell_p99"] <= e["per_cell_max"]


def test_algorithmic_bytes_of_the_configured_step():
    n, ncells = 10_000_000, 128 ** 3
    assert workload.algorithmic_bytes("mixed", n, ncells) == n * 76 + ncells * 36
    assert workload.algorithmic_bytes("fp64", n, ncells) == n * 104 + ncells * 48
    assert workload.step_kernel_bytes("mixed", n, ncells) == n * 76 + ncells * 12
    # 835 MB per step and 785 MB per step kernel at 1e7 parcels on 128^3 cells
    assert round(workload.algorithmic_bytes("mixed", n, ncells) / 1e6) == 835
    assert round(workload.step_kernel_bytes("mixed", n, ncells) / 1e6) == 785
    nt = 6 * 96 ** 3
    assert workload.tet_step_kernel_bytes("mixed", 20_000_000, nt) == 20_000_000 * 84 + nt * 156


def test_reference_arm_under_two_ranks_prints_one_line():
    """`bench.py --impl reference` launched by torchrun with two ranks: rank 0 alone times the
    reference's CPU path and prints one JSON line; the other rank exits 0 without output."""
    import json
    import socket
    import subprocess
    import sys

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--nparcels", "20000"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
