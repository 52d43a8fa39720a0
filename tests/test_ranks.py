"""The bench's multi-rank plumbing on CPU: two gloo ranks (spawned processes,
rendezvous on 127.0.0.1).  Every rank takes the slowest rank's time, the job
rate counts every rank's cells, and the reference arm prints on rank 0 only
while the other ranks exit without work."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as tdist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [3.0, 7.5][rank]
    slow = bench.max_over_ranks(ms, (torch, tdist))
    out.put((rank, slow, bench.job_rate(1000, 10, world, slow)))
    tdist.barrier()
    tdist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [7.5, 7.5]
    # 2 ranks x 1000 cells x 10 steps in 7.5 ms
    assert all(abs(r[2] - 2 * 1000 * 10 / 7.5e-3 / 1e6) < 1e-9 for r in res)


def test_max_over_ranks_single_process():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(4.25, None) == 4.25


def test_reference_arm_prints_on_rank_zero_only():
    # rank 1 of 2 exits at once with no output; rank 0 runs the bounded
    # CPU sample (a tiny one here) and prints the reference line
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    cmd = [sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--ref-cells", "40", "--cpu-steps", "2"]
    r1 = subprocess.run(cmd, env=dict(env, RANK="1", WORLD_SIZE="2"), capture_output=True, text=True, timeout=300,
                        cwd=ROOT)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r0.returncode == 0, r0.stderr
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
