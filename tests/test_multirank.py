"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1 reduce
their timings the way the GPU ranks do over NCCL (max of the times, sum of
the steps), each rank walks its own replica seed, and the reference arm does
its work on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: times 10+r and 20+2r ms, 1000*(r+1) steps, 500*(r+1) end-to-end steps
        res = bench.reduce_rank_times(dist, 10.0 + rank, 20.0 + 2 * rank, 1000 * (rank + 1), 500 * (rank + 1), "cpu")
        out[rank] = res + (bench.rank_seed(rank),)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_steps():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, ms2, steps, e2e = res[r][:4]
        assert (ms, ms2) == (11.0, 22.0)          # the slowest rank's times
        assert (steps, e2e) == (3000.0, 1500.0)   # every rank's steps
    assert res[0][4] != res[1][4]                 # one replica seed per rank


def test_single_process_passes_figures_through():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_rank_times(None, 5.0, 6.0, 7, 8, "cpu") == (5.0, 6.0, 7.0, 8.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference_arm(None, dict(bench.WORKLOADS["c1"])) == 0
