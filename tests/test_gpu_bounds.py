"""LB parity of the CUDA bound kernels with the reference (bit-exact int32)."""
import numpy as np
import pytest

from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", [None, 0, 1, 2])
def test_bound_children_vs_reference_golden(bounds_golden, method):
    """method None: the ABI entry point; 0: max-plus sweeps over all
    positions; 1: direct per-child scans and 2: sweeps, both over the free
    positions only, as the explorer runs them."""
    for case in bounds_golden["cases"]:
        p = np.array(case["p"], np.int32)
        nodes = case["nodes"]
        sched = np.array([nd["sched"] for nd in nodes], np.int32)
        l1 = np.array([nd["l1"] for nd in nodes], np.int32)
        l2 = np.array([nd["l2"] for nd in nodes], np.int32)
        g = pb.bound_children(p, sched, l1, l2, method=method)
        for i, nd in enumerate(nodes):
            assert (g["weak_begin"][i] == nd["weak_begin"]).all(), (case["n"], case["m"], i)
            assert (g["weak_end"][i] == nd["weak_end"]).all(), (case["n"], case["m"], i)
            assert (g["strong_begin"][i] == nd["strong_begin"]).all(), (case["n"], case["m"], i)
            assert (g["strong_end"][i] == nd["strong_end"]).all(), (case["n"], case["m"], i)
            assert g["node_weak"][i] == nd["node_weak"], (case["n"], case["m"], i)
            assert g["node_strong"][i] == nd["node_strong"], (case["n"], case["m"], i)


def random_nodes(rng, n, count):
    sched = np.stack([rng.permutation(n) for _ in range(count)]).astype(np.int32)
    nf = rng.integers(0, n, size=count)
    nb = np.array([rng.integers(0, n - f + 1) for f in nf])
    l1 = (nf - 1).astype(np.int32)
    l2 = (n - nb).astype(np.int32)
    keep = l1 < l2
    return sched[keep], l1[keep], l2[keep]


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("n,m,seed", [(20, 20, 1), (50, 20, 2), (33, 5, 7), (64, 20, 8), (9, 2, 9), (17, 32, 10)])
def test_bound_children_vs_oracle_random(n, m, seed, method):
    p = synthetic_instance(seed, n, m)
    O = Oracle(p)
    rng = np.random.default_rng(seed)
    sched, l1, l2 = random_nodes(rng, n, 300)
    g = pb.bound_children(p, sched, l1, l2, method=method)
    for i in range(len(sched)):
        cb, ce, _, _ = O.weak_children(sched[i], l1[i], l2[i])
        assert (g["weak_begin"][i] == cb).all()
        assert (g["weak_end"][i] == ce).all()
        assert (g["strong_begin"][i] == O.strong_children(sched[i], l1[i], l2[i], True)).all()
        assert (g["strong_end"][i] == O.strong_children(sched[i], l1[i], l2[i], False)).all()
        assert g["node_weak"][i] == O.weak_node(sched[i], l1[i], l2[i])
        assert g["node_strong"][i] == O.strong_node(sched[i], l1[i], l2[i])


@pytest.mark.parametrize("mode", [1, 2])
def test_johnson_pair_modes(mode):
    p = synthetic_instance(12, 24, 9)
    O = Oracle(p, pair_mode=mode)
    rng = np.random.default_rng(mode)
    sched, l1, l2 = random_nodes(rng, 24, 120)
    g = pb.bound_children(p, sched, l1, l2, johnson_mode=mode)
    for i in range(len(sched)):
        assert g["node_strong"][i] == O.strong_node(sched[i], l1[i], l2[i])
        assert (g["strong_begin"][i] == O.strong_children(sched[i], l1[i], l2[i], True)).all()


def test_lb_agreement_large_sample():
    """10^5 sampled nodes of the 50x20 instance (seed 2) against the oracle,
    itself pinned to the reference bounds library."""
    n, m = 50, 20
    p = synthetic_instance(2, n, m)
    O = Oracle(p)
    rng = np.random.default_rng(123)
    sched, l1, l2 = random_nodes(rng, n, 100000)
    g = pb.bound_children(p, sched, l1, l2)
    # the node-level Johnson and weak LBs of all nodes, children of a subsample
    want_s = np.array([O.strong_node(sched[i], l1[i], l2[i]) for i in range(len(sched))])
    want_w = np.array([O.weak_node(sched[i], l1[i], l2[i]) for i in range(len(sched))])
    assert (g["node_strong"] == want_s).all()
    assert (g["node_weak"] == want_w).all()
    for i in range(0, len(sched), 997):
        assert (g["strong_begin"][i] == O.strong_children(sched[i], l1[i], l2[i], True)).all()
        assert (g["strong_end"][i] == O.strong_children(sched[i], l1[i], l2[i], False)).all()


@pytest.mark.parametrize("n,m,seed", [(20, 20, 1), (50, 20, 2), (9, 4, 3)])
def test_bound_children_ex_priorities_and_idle(n, m, seed):
    """pbb_bound_children_ex: the weak bound's idle-time priorities of every
    child and the Johnson bound's couts[1] per node, bit-exact with the
    reference bounds library (the oracle when it is not built)."""
    import oracle
    p = synthetic_instance(seed, n, m)
    rng = np.random.default_rng(seed + 100)
    sched, l1, l2 = random_nodes(rng, n, 400)
    g = pb.bound_children_ex(p, sched, l1, l2)
    chk = oracle.Reference(p) if oracle.reference_available() else Oracle(p)
    O = Oracle(p)
    for i in range(len(sched)):
        _, _, pbw, pew = chk.weak_children(sched[i], l1[i], l2[i])
        free = sched[i, l1[i] + 1:l2[i]]
        assert (g["prio_begin"][i][free] == pbw[free]).all() and (g["prio_end"][i][free] == pew[free]).all()
        fixed = np.setdiff1d(np.arange(n), free)
        assert (g["prio_begin"][i][fixed] == 0).all() and (g["prio_end"][i][fixed] == 0).all()
        if isinstance(chk, oracle.Reference):
            want = chk.strong_node_idle(sched[i], l1[i], l2[i], unset=0)
        else:
            want = O.strong_node_idle(sched[i], l1[i], l2[i])
        assert g["strong_idle"][i] == want
        assert (g["weak_begin"][i] == O.weak_children(sched[i], l1[i], l2[i])[0]).all()
