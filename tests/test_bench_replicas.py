"""Host plumbing of bench.py's multi-GPU mode on CPU.

The solver does not shard (one mesh per GPU); `bench.py --gpus N` runs N
independent replicas and reports the max over ranks.  These tests run the
replica reduction as two gloo ranks and check that the CPU reference arm
only runs on rank 0.
"""
from __future__ import annotations

import datetime
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, ws: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        got = bench._dist()
        v = bench._barrier_max(1.5 * (rank + 1), ws, rank)
        q.put((rank, got, v))
    finally:
        dist.destroy_process_group()


def test_replica_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [(2, 0, 0), (2, 1, 1)]
    assert all(r[2] == 3.0 for r in res)


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"], env=env,
                         cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == ""
