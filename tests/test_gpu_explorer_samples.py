"""LB parity of the explorer's own bound code on nodes it actually bounded.

The explorer does not bound through pbb_bound_children: it keeps heads and
tails of the fixed jobs in a per-level path stack, scans the Johnson orders
over the free positions only, walks up to four children's scans together and
switches to max-plus sweeps for more children.  Here it records nodes as it
bounds them (hash of explorer id and step, include/pbbperm_diag.h), and every
recorded value is checked bit-exact against the reference's own bounds
library (oracle/_ref/libref_bounds.so: bound_fsp_weak::boundChildren, and
bound_fsp_strong::bornes_calculer on each child the explorer evaluated, as
ivm_bound::computeStrongBounds calls it, multicore/src/ivm_bound.cpp:141-195).
The side chosen and the set of Johnson-evaluated children are checked against
the reference's rules: MinMin (ivm_bound.cpp:479-504) on the weak bounds with
the incumbent as UB, and Johnson only for children the weak bound keeps on
that side (ivm_bound.cpp:168)."""
import numpy as np
import pytest

import oracle
from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

pytestmark = pytest.mark.gpu


def minmin_side(cb, ce, ub):
    """chooseChildrenSet rule 3 over (count, n) cost arrays (0 = fixed job)."""
    big = np.iinfo(np.int32).max
    mn = np.minimum(np.where(cb > 0, cb, big).min(axis=1), np.where(ce > 0, ce, big).min(axis=1))
    cnt = (cb == mn[:, None]).sum(axis=1) - (ce == mn[:, None]).sum(axis=1)
    elim = (cb >= ub[:, None]).sum(axis=1) - (ce >= ub[:, None]).sum(axis=1)
    return np.where(cnt > 0, 1, np.where(cnt < 0, 0, np.where(elim > 0, 0, 1)))


def collect(p, ub, ivms, cap, rate_log2, warm_s, mode=2):
    with pb.Engine(p, pb.Config(boundingMode=mode, adaptiveBranchingMode=3, nbIVMs=ivms)) as e:
        e.start(ub=ub)
        done = e.explore(warm_s) if warm_s > 0 else False
        e.sample_nodes(cap, rate_log2)
        for _ in range(4000):
            if done or e.sample_count() >= cap:
                break
            done = e.explore(0.02)
        return e.samples()


@pytest.mark.parametrize("n,m,seed,ivms,cap,rate,warm", [
    (50, 20, 2, 65536, 100000, 6, 0.5),    # the bench workload: UB = NEH, two-word rows
    (20, 20, 1, 16384, 30000, 7, 0.0),     # 20x20 at UB = optimum, one-word rows
])
def test_explorer_sampled_nodes_match_reference_bounds(n, m, seed, ivms, cap, rate, warm):
    p = synthetic_instance(seed, n, m)
    ub = pb.neh(p)[0] if n == 50 else 2352
    s = collect(p, ub, ivms, cap, rate, warm)
    cnt = len(s["k"])
    assert cnt >= (cap if n == 50 else cap // 2), cnt
    sched, l1, l2 = s["sched"], s["limit1"], s["limit2"]
    # records are well formed: permutations, limits consistent with the depth
    assert (np.sort(sched, axis=1) == np.arange(n)).all()
    assert ((l1 + 1) + (n - l2) == s["line"]).all() and (s["k"] == l2 - l1 - 1).all()
    wb, we, sb, se = s["weak_begin"], s["weak_end"], s["strong_begin"], s["strong_end"]
    free = np.zeros((cnt, n), bool)
    for i in range(cnt):
        free[i, sched[i, l1[i] + 1:l2[i]]] = True
    # side chosen: MinMin on the weak bounds with the incumbent as UB
    assert (s["side"] == minmin_side(wb, we, s["best"])).all()
    # Johnson evaluated exactly for the weak survivors on the chosen side
    keep_f = free & (wb < s["best"][:, None]) & (s["side"] == 0)[:, None]
    keep_b = free & (we < s["best"][:, None]) & (s["side"] == 1)[:, None]
    assert ((sb != 0) == keep_f).all() and ((se != 0) == keep_b).all()
    if oracle.reference_available():
        R = oracle.Reference(p)
        rwb, rwe, rsb, rse = R.children_batch(sched, l1, l2, sb != 0, se != 0)
        checked = cnt
    else:
        # without the reference build, the oracle (pinned to it by the golden
        # fixtures) checks a subsample
        O = Oracle(p)
        idx = np.arange(0, cnt, max(1, cnt // 2000))
        rwb, rwe, rsb, rse = [np.zeros((cnt, n), np.int32) for _ in range(4)]
        for i in idx:
            cb, ce, _, _ = O.weak_children(sched[i], l1[i], l2[i])
            rwb[i], rwe[i] = cb, ce
            rsb[i] = np.where(sb[i] != 0, O.strong_children(sched[i], l1[i], l2[i], True), 0)
            rse[i] = np.where(se[i] != 0, O.strong_children(sched[i], l1[i], l2[i], False), 0)
        sel = np.zeros(cnt, bool)
        sel[idx] = True
        wb, we, sb, se = [np.where(sel[:, None], a, 0) for a in (wb, we, sb, se)]
        checked = len(idx)
    for name, got, want in (("weak_begin", wb, rwb), ("weak_end", we, rwe), ("strong_begin", sb, rsb),
                            ("strong_end", se, rse)):
        bad = np.nonzero((got != want).any(axis=1))[0]
        assert len(bad) == 0, (name, len(bad), bad[:5].tolist())
    # the sample spans the tree: many depths and both scan regimes
    assert len(np.unique(s["line"])) >= 10
    assert checked > 0


def test_explorer_sampled_nodes_johnson_only_mode():
    """boundingMode 1 on the bench instance: the explorer evaluates the
    Johnson bound of every free child on both sides (computeStrongBounds
    without the weak pre-filter, ivm_bound.cpp:141-195), chooses the side by
    MinMin on those values, and each value equals the reference library's."""
    n, m = 50, 20
    p = synthetic_instance(2, n, m)
    ub = pb.neh(p)[0]
    s = collect(p, ub, 65536, 10000, 6, 0.5, mode=1)
    cnt = len(s["k"])
    assert cnt >= 10000, cnt
    sched, l1, l2 = s["sched"], s["limit1"], s["limit2"]
    assert (np.sort(sched, axis=1) == np.arange(n)).all()
    sb, se = s["strong_begin"], s["strong_end"]
    free = np.zeros((cnt, n), bool)
    for i in range(cnt):
        free[i, sched[i, l1[i] + 1:l2[i]]] = True
    assert ((sb != 0) == free).all() and ((se != 0) == free).all()
    assert (s["weak_begin"] == 0).all() and (s["weak_end"] == 0).all()
    assert (s["side"] == minmin_side(sb, se, s["best"])).all()
    if oracle.reference_available():
        _, _, rsb, rse = oracle.Reference(p).children_batch(sched, l1, l2, free, free)
        idx = np.arange(cnt)
    else:
        O = Oracle(p)
        idx = np.arange(0, cnt, max(1, cnt // 500))
        rsb, rse = np.zeros((cnt, n), np.int32), np.zeros((cnt, n), np.int32)
        for i in idx:
            rsb[i] = np.where(free[i], O.strong_children(sched[i], l1[i], l2[i], True), 0)
            rse[i] = np.where(free[i], O.strong_children(sched[i], l1[i], l2[i], False), 0)
    for name, got, want in (("strong_begin", sb, rsb), ("strong_end", se, rse)):
        bad = idx[(got[idx] != want[idx]).any(axis=1)]
        assert len(bad) == 0, (name, len(bad), bad[:5].tolist())
    assert len(np.unique(s["line"])) >= 10
