"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1 reduce
their timings the way the GPU ranks do over NCCL (max of the times, sum of
the steps), split one walker population into id shards, and combine the
shards' path-hash sums into the population's checksum; the reference arm
does its work on rank 0 only."""
import os
import socket
import sys

import numpy as np
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
        # each rank walks its shard of one population with the oracle
        from oracle import oracle as O
        beg, csr = O.rmat_graph(11, 8, seed=5)
        n = len(beg) - 1
        first, count = bench.rank_shard(rank, world, n)
        cfg = O.make_cfg(algo=0, maxhops=20, p=0.5, q=2.0, seed=42)
        h = O.walk(beg, csr, cfg, first, count, paths=False)["hashes"]
        local = int(h.sum(dtype=np.uint64))
        pop = bench.combine_hash_sums(dist, local, "cpu")
        out[rank] = res + ((first, count), pop)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_shard_walkers():
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
    # the shards tile the population, and their combined checksum is the
    # one-process checksum of the whole population
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    beg, csr = O.rmat_graph(11, 8, seed=5)
    n = len(beg) - 1
    (f0, c0), (f1, c1) = res[0][4], res[1][4]
    assert f0 == 0 and f0 + c0 == f1 and f1 + c1 == n
    whole = O.walk(beg, csr, O.make_cfg(algo=0, maxhops=20, p=0.5, q=2.0, seed=42), 0, n, paths=False)["hashes"]
    assert res[0][5] == res[1][5] == int(whole.sum(dtype=np.uint64))


@pytest.mark.parametrize("world,n", [(1, 10), (3, 10), (8, 3), (4, 1 << 20)])
def test_rank_shards_tile_the_population(world, n):
    sys.path.insert(0, ROOT)
    import bench
    shards = [bench.rank_shard(r, world, n) for r in range(world)]
    assert shards[0][0] == 0
    for (f, c), (g, _) in zip(shards, shards[1:]):
        assert f + c == g
    assert sum(c for _, c in shards) == n
    assert max(c for _, c in shards) - min(c for _, c in shards) <= 1


def test_single_process_passes_figures_through():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_rank_times(None, 5.0, 6.0, 7, 8, "cpu") == (5.0, 6.0, 7.0, 8.0)
    assert bench.combine_hash_sums(None, (1 << 64) + 5, "cpu") == 5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference_arm(None, dict(bench.WORKLOADS["c1"])) == 0
