"""The CPU oracle against the reference (no GPU).

Pins oracle/pbb_oracle.c to (1) the golden fixtures produced by the
reference's own bounds library and multicore B&B, (2) the reference's
testBounds known answers, and (3) the reference library itself when
oracle/_ref was built on this machine.
"""
import numpy as np
import pytest

import oracle
from oracle import Oracle
from pbbperm_b200.instances import synthetic_instance


def test_generator_matches_c():
    for seed, n, m in [(0, 20, 5), (1, 20, 20), (2, 50, 20), (99, 7, 3)]:
        assert (synthetic_instance(seed, n, m) == oracle.synthetic_instance(seed, n, m)).all()


def test_generator_range_and_shape():
    p = synthetic_instance(5, 40, 9)
    assert p.shape == (9, 40) and p.dtype == np.int32
    assert p.min() >= 1 and p.max() <= 99


def test_oracle_bounds_vs_golden(bounds_golden):
    checked = 0
    for case in bounds_golden["cases"]:
        p = np.array(case["p"], np.int32)
        O = Oracle(p)
        for s, row in enumerate(case["johnson"]):
            assert (O.johnson_row(s) == np.array(row)).all()
        for nd in case["nodes"]:
            sched = np.array(nd["sched"], np.int32)
            l1, l2 = nd["l1"], nd["l2"]
            cb, ce, _, _ = O.weak_children(sched, l1, l2)
            assert (cb == nd["weak_begin"]).all() and (ce == nd["weak_end"]).all()
            assert (O.strong_children(sched, l1, l2, True) == nd["strong_begin"]).all()
            assert (O.strong_children(sched, l1, l2, False) == nd["strong_end"]).all()
            assert O.weak_node(sched, l1, l2) == nd["node_weak"]
            assert O.strong_node(sched, l1, l2) == nd["node_strong"]
            assert O.eval(sched) == nd["makespan"]
            checked += 1
    assert checked > 300


def test_oracle_search_vs_golden(search_golden):
    """Node counters of the sequential restatement equal the reference
    multicore's at UB = optimum (small instances only; the rest run on GPU)."""
    done = 0
    for r in search_golden["runs"]:
        if r.get("ub") is None or r.get("big") or r["decomposed"] > 300000:
            continue
        p = synthetic_instance(r["seed"], r["n"], r["m"])
        got = Oracle(p).solve(r["ub"], bound_mode=r["bounding_mode"], branch_mode=r["branching_mode"],
                              find_all=r["find_all"])
        for k in ("decomposed", "johnson_bounds", "simple_bounds", "leaves"):
            assert got[k] == r[k], (r, k, got[k])
        done += 1
    assert done >= 20


def test_oracle_sorted_dfs_vs_golden(sorted_golden):
    """sortedDFS 0-4 from UB = +inf on one reference thread: the counters
    depend on the order children are explored in, so they pin the row
    reversal, the sort by the chosen side's first cost and the sorts by
    (cost, priority) and by priority for sortingCriterion 1-3."""
    KEYS = ("decomposed", "johnson_bounds", "simple_bounds", "leaves")
    for r in sorted_golden["runs"]:
        p = np.array(r["p"], np.int32)
        got = Oracle(p).solve(2**31 - 1, bound_mode=r["bounding_mode"], branch_mode=r["branching_mode"],
                              sorted_dfs=r["sorted_dfs"], sorting_criterion=r.get("sorting_criterion", 1))
        assert got["best"] == r["best"]
        for k in KEYS:
            assert got[k] == r[k], (r["seed"], r["bounding_mode"], r["branching_mode"], r["sorted_dfs"], k)


def test_oracle_weak_optimum_vs_golden(search_golden):
    for r in search_golden["runs"]:
        if r.get("ub") is None:
            p = synthetic_instance(r["seed"], r["n"], r["m"])
            O = Oracle(p)
            got = O.solve(2**31 - 1, bound_mode=r["bounding_mode"])
            assert got["best"] == r["opt"] and got["found"]
            assert O.eval(got["perm"]) == r["opt"]
            assert O.eval(np.array(r["perm"])) == r["opt"]


# testBounds known answers (bounds/test/testBounds.cpp:71-96 run on the
# reference build): makespan of the identity, LB1/LB2 at the root, LB1/LB2
# with the first and the last job fixed.
KNOWN = {1: (1448, 1232, 1278, 1297, 1297), 20: (2051, 1356, 1496, 1705, 1705)}


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("ta", sorted(KNOWN))
def test_testbounds_known_answers(ta):
    p = oracle.Reference.taillard(ta)
    m, n = p.shape
    O = Oracle(p)
    ident = np.arange(n, dtype=np.int32)
    got = (O.eval(ident), O.weak_node(ident, -1, n), O.strong_node(ident, -1, n),
           O.weak_node(ident, 0, n - 1), O.strong_node(ident, 0, n - 1))
    assert got == KNOWN[ta]


@pytest.mark.skipif(not oracle.reference_available(), reason="oracle/_ref not built")
def test_oracle_vs_reference_library_random_nodes():
    rng = np.random.default_rng(11)
    for n, m, seed in [(15, 4, 3), (27, 11, 4), (40, 16, 5)]:
        p = synthetic_instance(seed, n, m)
        O, R = Oracle(p), oracle.Reference(p)
        for _ in range(150):
            s = rng.permutation(n).astype(np.int32)
            nf = int(rng.integers(0, n)); nb = int(rng.integers(0, n - nf + 1))
            l1, l2 = nf - 1, n - nb
            if l1 >= l2:
                continue
            assert O.strong_node(s, l1, l2) == R.strong_node(s, l1, l2)
            assert O.weak_node(s, l1, l2) == R.weak_node(s, l1, l2)
            a, b = O.weak_children(s, l1, l2), R.weak_children(s, l1, l2)
            assert (a[0] == b[0]).all() and (a[1] == b[1]).all()


def test_neh_is_a_valid_upper_bound():
    for seed, n, m in [(0, 20, 5), (2, 50, 20)]:
        p = synthetic_instance(seed, n, m)
        O = Oracle(p)
        c, perm = O.neh()
        assert sorted(perm.tolist()) == list(range(n))
        assert O.eval(perm) == c
        assert c >= O.strong_node(np.arange(n), -1, n)


def test_oracle_priorities_and_idle_vs_reference_library():
    """The weak bound's idle-time priorities (prioBegin / prioEnd) and the
    Johnson bound's couts[1] of the oracle equal the reference bounds
    library's on random nodes (what pbb_bound_children_ex returns)."""
    if not oracle.reference_available():
        pytest.skip("reference checker not built")
    for seed, n, m in [(71, 12, 6), (72, 20, 20), (73, 33, 5)]:
        p = synthetic_instance(seed, n, m)
        O, R = Oracle(p), oracle.Reference(p)
        rng = np.random.default_rng(seed)
        for _ in range(60):
            s = rng.permutation(n).astype(np.int32)
            nf = int(rng.integers(0, n))
            nb = int(rng.integers(0, n - nf + 1))
            l1, l2 = nf - 1, n - nb
            if l1 >= l2:
                continue
            _, _, opb, ope = O.weak_children(s, l1, l2)
            _, _, rpb, rpe = R.weak_children(s, l1, l2)
            free = s[l1 + 1:l2]
            assert (opb[free] == rpb[free]).all() and (ope[free] == rpe[free]).all()
            want = R.strong_node_idle(s, l1, l2, unset=0)
            assert O.strong_node_idle(s, l1, l2) == want, (seed, l1, l2)
