"""Host logic of the multi-GPU path (polystokes_brownian_b200/shard.py), on CPU:
LPT partition properties, and world_size-2 gloo process groups for the per-rank
shares and the max/sum over ranks that bench.py uses."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from polystokes_brownian_b200 import configs, shard


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 100, size=257) ** 2)
    for n in (1, 2, 3, 8):
        parts = shard.lpt_partition(costs, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= (4/3 - 1/(3n)) OPT <= (4/3) * max(mean, max item)
        assert max(loads) <= (4 / 3) * max(sum(costs) / n, max(costs)) + 1e-9
    assert shard.lpt_partition([5.0, 5.0], 2) == [[0], [1]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = configs.ensemble(16, seed=3, nmin=32, nmax=256)
        mine = shard.rank_systems(systems, rank, world)
        ids = [s.name + str(int(s.x[0, 0] * 1e6)) for s in mine]
        local = float(sum(shard.replica_cost(s) for s in mine))
        out[rank] = (ids, local, shard.max_over_ranks(local), shard.sum_over_ranks(local))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shares_and_reductions():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    ids0, l0, m0, s0 = out[0]
    ids1, l1, m1, s1 = out[1]
    assert not set(ids0) & set(ids1)
    assert len(ids0) + len(ids1) == 16
    assert m0 == m1 == max(l0, l1)
    assert s0 == s1 == pytest.approx(l0 + l1)
