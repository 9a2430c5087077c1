"""Several GPUs on one search: disjoint factoradic intervals per rank.

Each rank explores its own intervals of [0, n!) with no data-path collective;
between windows the ranks exchange the incumbent (a 4-byte MIN all-reduce)
and, when a rank has run out of work, rebalance: the rank holding the most
work hands half of its intervals to the idle rank, point to point, and both
restart their explorers on the new intervals (pbb_init_from_fac).  This is
the role of the reference's master/worker interval exchange
(distributed/src/master.cpp, worker_gpu.cpp:33-60, work::split), restated
for ranks of one node: sizes are permutation counts, intervals travel as
factoradic digit vectors into the receiver's own memory.

Engines only need get_intervals() -> (pos, end, ids) and
init_from_fac(ub, pos, end, root=...); the CPU tests drive the same code with
a stand-in engine over gloo.
"""
import math

import numpy as np


def fact_index(d):
    """Permutation index of a factoradic vector: sum_i d_i (n-1-i)!."""
    n = len(d)
    v = 0
    for i in range(n):
        v = v * (n - i) + int(d[i])
    return v


def fact_digits(n, v):
    """Inverse of fact_index for 0 <= v < n!."""
    d = [0] * n
    for i in range(n - 1, -1, -1):
        v, d[i] = divmod(v, n - i)
    if v:
        raise ValueError("index not below n!")
    return d


def interval_load(pos, end):
    """Permutations covered by the intervals (inclusive ends)."""
    return sum(max(0, fact_index(e) - fact_index(p) + 1) for p, e in zip(pos, end))


def split_work(n, pos, end):
    """Split a rank's intervals into (keep, give), each a (pos, end) pair of
    lists, so that `give` holds about half of the permutations.  Several
    intervals: whole intervals from the end of the index order move until
    half is given; one interval [a, b]: it is cut at its middle."""
    iv = sorted(((fact_index(p), fact_index(e)) for p, e in zip(pos, end)), key=lambda x: x[0])
    iv = [(a, b) for a, b in iv if a <= b]
    total = sum(b - a + 1 for a, b in iv)
    keep, give = list(iv), []
    if len(iv) == 1:
        a, b = iv[0]
        if b > a:
            mid = (a + b) // 2
            keep, give = [(a, mid)], [(mid + 1, b)]
    else:
        given = 0
        while len(keep) > 1 and given * 2 < total:
            a, b = keep.pop()
            give.insert(0, (a, b))
            given += b - a + 1

    def unpack(lst):
        return [fact_digits(n, a) for a, _ in lst], [fact_digits(n, b) for _, b in lst]

    return unpack(keep), unpack(give)


def plan_rebalance(loads):
    """(donor, receiver) pairs: every idle rank (load 0) is matched with a
    distinct rank holding work, the largest loads first; a donor's load must
    be at least 2 (something to split).  Deterministic, so every rank
    computes the same plan from the same gathered loads."""
    idle = [r for r, x in enumerate(loads) if x <= 0]
    donors = sorted((r for r, x in enumerate(loads) if x >= 2), key=lambda r: (-loads[r], r))
    return list(zip(donors, idle))


def rebalance(dist, eng, n, ub, root, device="cpu", done=False):
    """One rebalancing step between windows, on every rank (same collective
    sequence everywhere).  Returns True when this rank restarted its engine
    on new intervals (its counters restart from zero)."""
    import torch

    rank, world = dist.get_rank(), dist.get_world_size()
    if done:
        pos, end = [], []
    else:
        p, e, _ = eng.get_intervals()
        pos, end = [list(x) for x in p], [list(x) for x in e]
    # planning load: the number of intervals (an explorer holding work holds
    # one), or for a single interval whether it can be cut (2) or not (1);
    # exact sizes are only computed by a donor when it splits
    load = len(pos)
    if load == 1:
        load = 2 if interval_load(pos, end) >= 2 else 1
    t = torch.tensor([float(load)], dtype=torch.float64, device=device)
    loads = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(loads, t)
    plan = plan_rebalance([x.item() for x in loads])
    changed = False
    for donor, receiver in plan:
        if rank == donor:
            (kp, ke), (gp, ge) = split_work(n, pos, end)
            cnt = torch.tensor([len(gp)], dtype=torch.int32, device=device)
            dist.send(cnt, receiver)
            if gp:
                dist.send(torch.tensor(np.array(gp + ge, np.int32), device=device), receiver)
                eng.init_from_fac(ub, np.array(kp, np.int32), np.array(ke, np.int32), root=root)
                changed = True
        elif rank == receiver:
            cnt = torch.zeros(1, dtype=torch.int32, device=device)
            dist.recv(cnt, donor)
            k = int(cnt.item())
            if k:
                buf = torch.zeros((2 * k, n), dtype=torch.int32, device=device)
                dist.recv(buf, donor)
                a = buf.cpu().numpy()
                eng.init_from_fac(ub, a[:k].copy(), a[k:].copy(), root=root)
                changed = True
    return changed


def total_permutations(n):
    return math.factorial(n)
