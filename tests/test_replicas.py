"""The multi-GPU form is replicas only (no data-path collective): N ranks
each apply the operator, and bench.py reports the whole job's rate from the
slowest rank (max over ranks). These tests run that host logic as two gloo
ranks on the CPU: the barrier, the max over ranks and the replica rate."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup(backend="gloo")
    try:
        bench.barrier(w)
        # rank r took 10 + 5 r ms for 4 applies
        value, ms_total = bench.replica_rate(10.0 + 5.0 * r, 4, w, torch.device("cpu"))
        out.put((r, w, local, value, ms_total))
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(out.get(timeout=5) for _ in range(2))
    for r, (rank, world, local, value, ms_total) in enumerate(res):
        assert (rank, world, local) == (r, 2, r)
        assert ms_total == pytest.approx(15.0)            # the slower rank's time, on every rank
        assert value == pytest.approx(2 * 4 / 0.015)      # whole-job applies per second


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    import torch
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        assert bench.dist_setup(backend="gloo") == (1, 0, 0)
        assert bench.replica_rate(20.0, 5, 1, torch.device("cpu")) == (250.0, 20.0)
    finally:
        os.environ.update(env)
