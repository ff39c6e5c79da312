"""Multi-process host logic on the CPU (gloo, world size 2): bench.py's replica reduction takes
the slowest rank's time and the sum of the ranks' work, and the reference arm runs on rank 0
only. No simulation data crosses ranks (replicas only)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    ms, work = bench.reduce_over_ranks(10.0 + rank * 5.0, 100.0 * (rank + 1), dist, "cpu")
    out[rank] = (ms, work)
    dist.barrier()
    dist.destroy_process_group()


def test_replica_reduction_two_ranks():
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0] == (15.0, 300.0) and out[1] == (15.0, 300.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        size, steps, warmup, cpu_seconds, precision = 64, 1, 1, 0.1, "f64"
    assert bench.run_reference(A()) == 0
    assert capsys.readouterr().out == ""
