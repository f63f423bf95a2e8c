"""The multi-GPU path of the benchmark is N independent replicas: the only
cross-rank steps are a barrier and the max-time / sum-of-events reduction.
Checked here with world_size 2 over gloo on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world)
    # rank r ran for (r + 1) s and delivered 10 * (r + 1) events
    t, e = bench.reduce_max_sum(world, float(rank + 1), 10.0 * (rank + 1))
    out.put((rank, t, e))
    bench.barrier(world)
    dist.destroy_process_group()


def test_replica_reduction_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest replica's time and the total work
    assert res == [(0, 2.0, 30.0), (1, 2.0, 30.0)]


def test_reference_arm_other_ranks_exit_quietly(capsys, monkeypatch):
    """Under torchrun only rank 0 times the reference's CPU step."""
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference"])
    args = bench.parse()
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
