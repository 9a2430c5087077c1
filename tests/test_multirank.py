"""The N>1 path of bench.py on CPU: root-level slices partition the search
space, and the incumbent exchange is a MIN all-reduce (gloo, world size 2)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def test_rank_slices_partition_root_level():
    for n in (2, 5, 20, 50, 64):
        for world in (1, 2, 3, 4, 8):
            if world == 1:
                assert bench.rank_slice(n, 0, 1) is None
                continue
            cells = []
            for r in range(world):
                sl = bench.rank_slice(n, r, world)
                if sl is None:
                    continue
                pos, end = sl
                assert len(pos) == n and len(end) == n
                assert all(0 <= pos[i] < n - i and 0 <= end[i] < n - i for i in range(n))
                assert pos[1:] == [0] * (n - 1) and end[1:] == [n - 1 - i for i in range(1, n)]
                cells += list(range(pos[0], end[0] + 1))
            assert cells == list(range(n)), (n, world)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.exchange_incumbent(dist, costs[rank], "cpu")
    finally:
        dist.destroy_process_group()


def test_incumbent_exchange_gloo_world2():
    world = 2
    costs = [4029, 3991]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), costs, out), nprocs=world, join=True)
    assert [out[r] for r in range(world)] == [min(costs)] * world
