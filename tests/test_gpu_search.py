"""The persistent IVM explorer against the reference: exact node counters at
UB = optimum, exact optima re-verified from the returned permutation."""
import numpy as np
import pytest

from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

pytestmark = pytest.mark.gpu

KEYS = ("decomposed", "johnson_bounds", "simple_bounds", "leaves")


def solve(p, ub, ivms=1024, **cfg):
    with pb.Engine(p, pb.Config(nbIVMs=ivms, **cfg)) as e:
        return e.solve(ub=ub)


def test_sorted_dfs_sequential_vs_reference_golden(sorted_golden):
    """One explorer from UB = +inf explores in the reference's sequential order,
    so its counters, which depend on when the bound improves, must equal the
    reference's single-thread run, with the rows reversed (sortedDFS = 0),
    sorted by the chosen side's bound (1), by (bound, priority) (2, 4) or by
    the priority (3), with and without the early Johnson exit."""
    for r in sorted_golden["runs"]:
        p = np.array(r["p"], np.int32)
        got = solve(p, 2**31 - 1, ivms=1, boundingMode=r["bounding_mode"],
                    adaptiveBranchingMode=r["branching_mode"], sortedDFS=r["sorted_dfs"],
                    sortingCriterion=r.get("sorting_criterion", 1), earlyStopJohnson=r.get("early_stop", False))
        assert got["complete"] and got["found"] and got["cost"] == r["best"]
        for k in KEYS:
            assert got[k] == r[k], (r["seed"], r["bounding_mode"], r["branching_mode"], r["sorted_dfs"], k,
                                    got[k], r[k])


@pytest.mark.parametrize("sorted_dfs,crit", [(2, 2), (3, 3), (4, 1)])
def test_priority_sorts_at_the_optimum_many_explorers(sorted_dfs, crit):
    """At UB = optimum the node set does not depend on the order: sortedDFS
    2-4 with 16384 explorers give the oracle's counters."""
    p = synthetic_instance(24, 13, 20)
    want = Oracle(p).solve(1803, bound_mode=2, sorted_dfs=sorted_dfs, sorting_criterion=crit)
    got = solve(p, 1803, ivms=16384, boundingMode=2, sortedDFS=sorted_dfs, sortingCriterion=crit)
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.parametrize("ivms", [64, 16384])
def test_sorted_dfs_counters_at_the_optimum(ivms):
    """At UB = optimum the node set does not depend on the order, with any
    number of explorers: counters equal the oracle's with the same sort."""
    p = synthetic_instance(24, 13, 20)
    want = Oracle(p).solve(1803, bound_mode=2, sorted_dfs=1)
    got = solve(p, 1803, ivms=ivms, boundingMode=2, sortedDFS=1)
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_counters_vs_reference_golden(search_golden):
    for r in search_golden["runs"]:
        if r.get("ub") is None or r.get("big"):
            continue
        p = synthetic_instance(r["seed"], r["n"], r["m"])
        got = solve(p, r["ub"], boundingMode=r["bounding_mode"], adaptiveBranchingMode=r["branching_mode"],
                    findAll=r["find_all"], earlyStopJohnson=r.get("early_stop", False))
        assert got["complete"]
        for k in KEYS:
            assert got[k] == r[k], (r, k, got[k])


@pytest.mark.parametrize("n,m,seed,mode", [(10, 5, 21, 2), (12, 10, 22, 1), (14, 5, 23, 0), (13, 20, 24, 2),
                                           (35, 10, 45, 0), (35, 10, 45, 2), (2, 3, 33, 2), (3, 2, 34, 1),
                                           (9, 32, 35, 2), (16, 8, 25, 2)])
def test_counters_vs_oracle(n, m, seed, mode):
    p = synthetic_instance(seed, n, m)
    O = Oracle(p)
    opt = O.solve(2**31 - 1, bound_mode=2)["best"]
    want = O.solve(opt, bound_mode=mode)
    got = solve(p, opt, boundingMode=mode)
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.parametrize("mode", [0, 2])
def test_counters_50x20_below_optimum(mode):
    """50x20 seed 2 with UB = 3780 (no schedule reaches it, so the search is
    deterministic): two-word IVM rows, 65536 explorers."""
    p = synthetic_instance(2, 50, 20)
    want = Oracle(p).solve(3780, bound_mode=mode)
    assert want["complete"] and not want["found"]
    got = solve(p, 3780, ivms=65536, boundingMode=mode)
    assert got["complete"] and not got["found"]
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_counters_64_jobs_without_kept_masks():
    """64 jobs x 20 machines: the tables leave no room for the per-warp
    free-position masks at the largest warp count, so the engine runs the
    general explorer build, which rebuilds each pair's mask at every node.
    UB = 4421 lies below every schedule (the oracle finds none), so the
    search is deterministic: counters equal the oracle's."""
    import torch
    p = synthetic_instance(5, 64, 20)
    want = Oracle(p).solve(4421, bound_mode=2)
    assert want["complete"] and not want["found"] and want["decomposed"] > 10000
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    with pb.Engine(p, pb.Config(nbIVMs=16384, boundingMode=2)) as e:
        got = e.solve(ub=4421)
        warps = e.kernel_stats()["warps"]          # all CTAs' warps; one CTA per SM
    assert warps // sms < 20, (warps, sms)
    assert got["complete"] and not got["found"]
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.parametrize("ivms", [1, 3, 64, 4096, 65536])
def test_counters_independent_of_explorer_count(ivms):
    p = synthetic_instance(24, 13, 20)
    O = Oracle(p)
    opt = 1803
    want = O.solve(opt, bound_mode=2)
    got = solve(p, opt, ivms=ivms, boundingMode=2)
    for k in KEYS:
        assert got[k] == want[k], (ivms, k, got[k], want[k])


@pytest.mark.parametrize("share_after", [-1, 1, 64, 5000])
def test_counters_independent_of_share_threshold(share_after):
    """How long an explorer works before it may hand work away changes who
    explores what, never which nodes are decomposed: counters equal the
    oracle's whether explorers split at every step (-1), after every node,
    after 64 (the default) or almost never."""
    p = synthetic_instance(24, 13, 20)
    want = Oracle(p).solve(1803, bound_mode=2)
    got = solve(p, 1803, ivms=4096, boundingMode=2, share_after=share_after)
    for k in KEYS:
        assert got[k] == want[k], (share_after, k, got[k], want[k])


def test_windowed_exploration_matches_single_solve():
    p = synthetic_instance(24, 13, 20)
    want = Oracle(p).solve(1803, bound_mode=2)
    with pb.Engine(p, pb.Config(nbIVMs=2048, boundingMode=2)) as e:
        e.start(ub=1803)
        done = False
        windows = 0
        while not done and windows < 10000:
            done = e.explore(0.002)
            windows += 1
        got = e.result()
    assert got["complete"]
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_weak_bound_optimum_ub_inf(search_golden):
    """20x5 seed 0, weak bound, UB = +inf: optimum equals the reference's and
    is re-verified from the returned permutation."""
    ref = [r for r in search_golden["runs"] if r.get("ub") is None][0]
    p = synthetic_instance(ref["seed"], ref["n"], ref["m"])
    got = solve(p, pb.INF, ivms=4096, boundingMode=0)
    assert got["complete"] and got["found"]
    assert got["cost"] == ref["opt"]
    assert Oracle(p).eval(got["perm"]) == ref["opt"]
    assert sorted(got["perm"].tolist()) == list(range(ref["n"]))


def test_optimum_found_from_ub_plus_one():
    p = synthetic_instance(22, 12, 10)
    got = solve(p, 1012, boundingMode=2)
    assert got["found"] and got["cost"] == 1011
    assert Oracle(p).eval(got["perm"]) == 1011


def test_root_permutation_respected():
    p = synthetic_instance(23, 14, 5)
    O = Oracle(p)
    root = np.random.default_rng(4).permutation(14).astype(np.int32)
    want = O.solve(862, bound_mode=2, root=root)
    with pb.Engine(p, pb.Config(nbIVMs=256, boundingMode=2)) as e:
        got = e.solve(ub=862, root=root)
    for k in KEYS:
        assert got[k] == want[k]


def test_config2_20x20_johnson_ub_opt(config2_golden):
    """20 jobs x 20 machines (seed 1), weak+Johnson bound, 16384 explorers,
    UB = optimum 2352: decomposed-node count equals the reference's."""
    c = config2_golden
    p = synthetic_instance(c["seed"], c["n"], c["m"])
    for share_after in (0, -1):
        got = solve(p, c["opt"], ivms=16384, boundingMode=2, share_after=share_after)
        assert got["complete"]
        for k in KEYS:
            assert got[k] == c[k], (share_after, k, got[k], c[k])


@pytest.mark.parametrize("world", [2, 3])
def test_interval_start_matches_oracle(world):
    """pbb_start_interval (gpubb::initAtInterval) on each rank's root slice:
    per-slice counters equal the oracle's interval solve, and the best of the
    slices is the optimum."""
    import bench
    p = synthetic_instance(24, 13, 20)
    O = Oracle(p)
    found = []
    for r in range(world):
        pos, end = bench.rank_slice(13, r, world)
        want = O.solve(1804, bound_mode=2, pos=pos, end=end)
        with pb.Engine(p, pb.Config(nbIVMs=1024, boundingMode=2)) as e:
            e.start_interval(ub=1804, pos=pos, end=end)
            while not e.explore(1.0):
                pass
            got = e.result()
        assert got["complete"]
        if want["found"]:
            assert got["found"] and got["cost"] == want["best"]
            found.append(got["cost"])
        else:
            for k in KEYS:
                assert got[k] == want[k], (r, k, got[k], want[k])
    assert min(found) == 1803
