"""The N>1 path on CPU (gloo): root-level slices partition the search space,
the incumbent exchange is a MIN all-reduce, and rebalancing moves half of the
busiest rank's intervals to an idle rank without gap or overlap."""
import os
import socket

import numpy as np

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


class _StandInEngine:
    """The two engine calls rebalancing uses, over host arrays."""

    def __init__(self, n, pos, end):
        self.n = n
        self.pos = np.array(pos, np.int32).reshape(-1, n)
        self.end = np.array(end, np.int32).reshape(-1, n)

    def get_intervals(self):
        return self.pos, self.end, np.arange(len(self.pos), dtype=np.int32)

    def init_from_fac(self, ub, pos, end, ids=None, root=None):
        self.pos = np.asarray(pos, np.int32).reshape(-1, self.n)
        self.end = np.asarray(end, np.int32).reshape(-1, self.n)


def _rebalance_worker(rank, world, port, n, work, out):
    from pbbperm_b200 import distributed as pd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pos, end = work[rank]
        eng = _StandInEngine(n, pos, end)
        changed = pd.rebalance(dist, eng, n, 1000, list(range(n)), device="cpu", done=len(pos) == 0)
        p, e, _ = eng.get_intervals() if len(eng.pos) else ([], [], [])
        out[rank] = (changed, [(pd.fact_index(a), pd.fact_index(b)) for a, b in zip(p, e)])
    finally:
        dist.destroy_process_group()


def _covered(intervals):
    cells = []
    for a, b in intervals:
        cells.extend(range(a, b + 1))
    return cells


@pytest.mark.parametrize("world,case", [(2, "one"), (2, "many"), (3, "one"), (4, "many")])
def test_rebalance_keeps_a_partition_gloo(world, case):
    """An idle rank receives half of the busiest rank's work; afterwards the
    ranks' intervals still cover exactly the same permutations, without
    overlap, and the idle ranks hold work."""
    from pbbperm_b200 import distributed as pd
    n = 6
    if case == "one":
        busy = [([0] * n, [n - 1 - i for i in range(n)])]                       # the whole space
    else:
        cuts = [0, 37, 200, 411, 650, 719]
        busy = [(pd.fact_digits(n, a), pd.fact_digits(n, b - 1)) for a, b in zip(cuts[:-1], cuts[1:])]
    work = [([p for p, _ in busy], [e for _, e in busy])] + [([], [])] * (world - 1)
    before = sorted(_covered([(pd.fact_index(p), pd.fact_index(e)) for p, e in busy]))
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rebalance_worker, args=(world, _free_port(), n, work, out), nprocs=world, join=True)
    after = []
    for r in range(world):
        after += _covered(out[r][1])
    assert sorted(after) == before                    # no gap, no overlap
    assert out[0][0] and out[1][0] and len(out[1][1]) > 0


def test_split_work_halves():
    from pbbperm_b200 import distributed as pd
    n = 7
    (kp, ke), (gp, ge) = pd.split_work(n, [[0] * n], [[n - 1 - i for i in range(n)]])
    k, g = pd.interval_load(kp, ke), pd.interval_load(gp, ge)
    assert k + g == 5040 and abs(k - g) <= 1
    assert pd.plan_rebalance([0, 10, 3, 0, 1]) == [(1, 0), (2, 3)]
