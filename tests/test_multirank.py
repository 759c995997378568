"""The multi-rank plumbing of bench.py on CPU: world size 2 over gloo, as torchrun launches it.

Replicas exchange nothing on the data path; the ranks only meet in barriers and in the timing
reduction (max of the per-rank times, sum of the queries), and the reference arm runs on rank 0
alone."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    r, w = bench.dist_init("gloo")
    bench.barrier(w)
    max_ms, total_q = bench.aggregate(1.5 + rank, 100 * (rank + 1), w)
    bench.barrier(w)
    out.put((r, w, max_ms, total_q, bench.replica_seed(7, r)))
    dist.destroy_process_group()


def test_timing_reduction_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    # every rank sees the slowest rank's time and the queries of both
    assert all(g[2] == 2.5 and g[3] == 300 for g in got)
    # each replica indexes its own data
    assert got[0][4] != got[1][4]


def test_reference_arm_runs_on_rank_zero_only():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--rows", "20000", "--dims", "64", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
