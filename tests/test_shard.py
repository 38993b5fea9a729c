"""Sharding of independent meshes across ranks (mmcuda.shard): the
partition covers every mesh exactly once, is balanced, and two gloo ranks
that compute it independently agree (the multi-GPU batched path has no
data-path collective, so this agreement is all it needs)."""
import os
import socket
import sys

import numpy as np
import pytest

from mmcuda.shard import padded_len, partition, step_cost

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_padded_lengths():
    # smallest 7-smooth >= 2n-1, even along x (the demag plan's padding)
    assert [padded_len(n) for n in (1, 2, 3, 64, 251, 256)] == [1, 3, 5, 128, 504, 512]
    assert padded_len(1000, even=True) == 2000 and padded_len(50, even=True) == 100


@pytest.mark.parametrize("nranks", [1, 2, 3, 8])
def test_partition_complete_and_balanced(nranks):
    rng = np.random.default_rng(1)
    costs = list(rng.uniform(1, 100, 48))
    parts = partition(costs, nranks)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(48))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "micromagnetic.jl_b200"))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    specs = bench.batch_specs("c3")
    mine = partition([step_cost(s["nx"], s["ny"], s["nz"]) for s in specs], world)[rank]
    t = torch.full((48,), -1, dtype=torch.int64)
    t[: len(mine)] = torch.tensor(mine, dtype=torch.int64)
    got = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(got, t)
    if rank == 0:
        lists = [[int(v) for v in g if v >= 0] for g in got]
        out.put(lists)
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_c3_partition():
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    lists = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(lists[0] + lists[1]) == list(range(48))
    assert not set(lists[0]) & set(lists[1])
