"""Initial bounds computed on the device: NEH (fastNEH's insertion
procedure, heuristic/src/fastNEH.cpp:206-243) one warp per instance, equal
job for job to the host restatement pbb_neh on every instance of the batched
and served workloads and on the benchmark instances."""
import numpy as np
import pytest

from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance, batch_instance, serving_instance

pytestmark = pytest.mark.gpu


def test_device_neh_equals_host_neh_on_the_workloads():
    insts = [batch_instance(100 + i) for i in range(512)]
    insts += [serving_instance(10000 + i) for i in range(256)]
    insts += [synthetic_instance(2, 50, 20), synthetic_instance(1, 20, 20), synthetic_instance(0, 20, 5),
              synthetic_instance(8, 64, 20), synthetic_instance(9, 7, 32), synthetic_instance(10, 2, 2),
              synthetic_instance(11, 3, 1), synthetic_instance(12, 1, 4)]
    got = pb.neh_batch(insts)
    for p, (cost, perm) in zip(insts, got):
        hc, hp = pb.neh(p)
        assert cost == hc and (perm == hp).all(), (p.shape, cost, hc)
        assert sorted(perm.tolist()) == list(range(p.shape[1]))


def test_device_neh_equals_oracle_neh():
    for seed, n, m in [(0, 20, 5), (2, 50, 20), (31, 33, 7)]:
        p = synthetic_instance(seed, n, m)
        (cost, perm), = pb.neh_batch([p])
        oc, operm = Oracle(p).neh()
        assert cost == oc and (perm == operm).all()
        assert Oracle(p).eval(perm) == cost


def test_engine_starts_from_device_neh():
    """PBB_UB_NEH: the engine computes NEH on the device and searches below
    it; the result is the optimum with a schedule, whether or not a leaf
    improved on NEH."""
    for seed, n, m in [(22, 12, 10), (21, 10, 5), (25, 16, 8), (26, 9, 4)]:
        p = synthetic_instance(seed, n, m)
        O = Oracle(p)
        opt = O.solve(2**31 - 1, bound_mode=2)["best"]
        with pb.Engine(p, pb.Config(boundingMode=2, nbIVMs=1024)) as e:
            got = e.solve(ub=pb.UB_NEH)
        assert got["complete"] and got["has_perm"] and got["cost"] == opt
        assert O.eval(got["perm"]) == opt
        neh_cost = pb.neh(p)[0]
        if neh_cost == opt:
            # nothing improves on NEH: the search is deterministic, and its
            # counters are those of a search from the NEH makespan
            want = O.solve(neh_cost, bound_mode=2)
            assert not got["found"]
            for k in ("decomposed", "johnson_bounds", "simple_bounds", "leaves"):
                assert got[k] == want[k], (seed, k, got[k], want[k])
        else:
            assert got["found"]


def test_pool_admits_with_device_neh():
    rng = np.random.default_rng(41)
    insts = [synthetic_instance(900 + i, int(rng.integers(8, 13)), int(rng.choice([3, 5, 8, 10]))) for i in range(48)]
    res = pb.batch_solve(insts, ubs=[pb.UB_NEH] * len(insts), config=pb.Config(boundingMode=2),
                         pool_config=pb.PoolConfig(max_jobs=12, max_machines=10, window_s=0.01))
    for p, r in zip(insts, res):
        opt = Oracle(p).solve(pb.neh(p)[0] + 1, bound_mode=2)["best"]
        assert r["complete"] and r["has_perm"] and r["cost"] == opt
        assert Oracle(p).eval(r["perm"]) == opt


@pytest.mark.parametrize("iterations", [0, 1, 25])
def test_device_ig_equals_its_restatement(iterations):
    """Seeded IG (heuristic/src/IG.cpp:341-416 with a splitmix64 stream): the
    device run equals the host restatement draw for draw, never exceeds NEH
    and returns a schedule of its makespan."""
    insts = [synthetic_instance(2, 50, 20), synthetic_instance(1, 20, 20), synthetic_instance(0, 20, 5),
             synthetic_instance(44, 12, 10), synthetic_instance(45, 3, 4), synthetic_instance(46, 64, 6)]
    insts += [batch_instance(100 + i) for i in range(10)]
    seed = 1234
    got = pb.ig_batch(insts, iterations=iterations, seed=seed)
    for t, (p, (cost, perm)) in enumerate(zip(insts, got)):
        O = Oracle(p)
        hc, hp = O.ig(iterations, seed + t)
        assert cost == hc and (perm == hp).all(), (t, p.shape, cost, hc)
        assert O.eval(perm) == cost
        assert cost <= pb.neh(p)[0]
        assert sorted(perm.tolist()) == list(range(p.shape[1]))
