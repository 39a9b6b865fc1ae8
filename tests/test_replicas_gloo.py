"""The multi-process path of bench.py on the CPU: two ranks over gloo (the
GPU path uses NCCL with one process per GPU).  The replicas share no data;
the process group only takes the slowest rank's time, and the whole-job
throughput counts every rank's work over that time."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, ws: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(ws), RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    w, r, local = bench.dist_init(backend="gloo")
    assert (w, r) == (ws, rank)
    t_local = 0.5 + 0.25 * rank          # rank 1 is the slower one
    t_max = bench.max_over_ranks(t_local, local)
    value = bench.replica_value(1000.0, t_max, w)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, t_max, value))


def test_two_replicas_take_the_slowest_rank_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [0.75, 0.75]
    assert all(abs(r[2] - 2000.0 / 0.75) < 1e-9 for r in res)


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(1.25) == 1.25
    assert bench.replica_value(10.0, 2.0, 1) == 5.0
