"""Batched and served solving through the resident pool: every instance's
result is the same in the mix as alone (exact counters at UB = optimum,
exact optima at UB = +inf), whatever the admission order."""
import numpy as np
import pytest

from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

pytestmark = pytest.mark.gpu

KEYS = ("decomposed", "johnson_bounds", "simple_bounds", "leaves")


def mixed_instances(count, seed0=300):
    rng = np.random.default_rng(seed0)
    out = []
    for i in range(count):
        n = int(rng.integers(8, 13))
        m = int(rng.choice([3, 5, 8, 10]))
        out.append(synthetic_instance(seed0 + i, n, m))
    return out


@pytest.fixture(scope="module")
def mix():
    insts = mixed_instances(40)
    ref = []
    for p in insts:
        O = Oracle(p)
        opt = O.solve(2**31 - 1, bound_mode=2)["best"]
        ref.append(dict(opt=opt, counts=O.solve(opt, bound_mode=2)))
    return insts, ref


@pytest.mark.parametrize("share_after", [0, -1, 16])
def test_batch_counters_equal_solo(mix, share_after):
    insts, ref = mix
    res = pb.batch_solve(insts, ubs=[r["opt"] for r in ref], config=pb.Config(boundingMode=2),
                         pool_config=pb.PoolConfig(max_jobs=12, max_machines=10, window_s=0.01,
                                                   share_after=share_after))
    for i, (got, r) in enumerate(zip(res, ref)):
        assert got["complete"]
        for k in KEYS:
            assert got[k] == r["counts"][k], (i, k, got[k], r["counts"][k])


def test_batch_optima_from_infinity(mix):
    insts, ref = mix
    res = pb.batch_solve(insts, config=pb.Config(boundingMode=2),
                         pool_config=pb.PoolConfig(max_jobs=12, max_machines=10, window_s=0.01,
                                                   explorers_per_instance=4096))
    for p, got, r in zip(insts, res, ref):
        assert got["found"] and got["cost"] == r["opt"]
        assert Oracle(p).eval(got["perm"]) == r["opt"]


def test_staggered_submission_matches_solo(mix):
    """Requests arrive while others are on the GPU (few resident slots force
    queueing and admission as slots free up)."""
    insts, ref = mix
    cfg = pb.PoolConfig(max_jobs=12, max_machines=10, max_resident=7, window_s=0.002)
    got = {}
    with pb.Pool(cfg) as pool:
        nxt = 0
        steps = 0
        while len(got) < len(insts) and steps < 100000:
            for _ in range(3):
                if nxt < len(insts):
                    pool.submit(insts[nxt], tag=nxt, ub=ref[nxt]["opt"], config=pb.Config(boundingMode=2))
                    nxt += 1
            pool.step()
            steps += 1
            for r in pool.poll():
                got[r["tag"]] = r
    assert len(got) == len(insts)
    for i, r in enumerate(ref):
        for k in KEYS:
            assert got[i][k] == r["counts"][k], (i, k)


def test_mixed_search_settings_in_one_pool(mix):
    insts, ref = mix
    modes = [0, 1, 2]
    want = []
    for i, p in enumerate(insts[:12]):
        want.append(Oracle(p).solve(ref[i]["opt"], bound_mode=modes[i % 3]))
    got = {}
    with pb.Pool(pb.PoolConfig(max_jobs=12, max_machines=10, window_s=0.005)) as pool:
        for i, p in enumerate(insts[:12]):
            pool.submit(p, tag=i, ub=ref[i]["opt"], config=pb.Config(boundingMode=modes[i % 3]))
        for _ in range(100000):
            res, q = pool.step()
            for r in pool.poll():
                got[r["tag"]] = r
            if res == 0 and q == 0:
                break
    for i in range(12):
        for k in KEYS:
            assert got[i][k] == want[i][k], (i, modes[i % 3], k)


def test_pool_two_word_rows():
    """Instances over 32 jobs use 64-byte rows (second kernel variant)."""
    p = synthetic_instance(45, 35, 10)
    O = Oracle(p)
    opt = O.solve(2**31 - 1, bound_mode=2)["best"]
    want = O.solve(opt, bound_mode=2)
    res = pb.batch_solve([p, synthetic_instance(22, 12, 10)], ubs=[opt, 1011], config=pb.Config(boundingMode=2),
                         pool_config=pb.PoolConfig(max_jobs=40, max_machines=10))
    for k in KEYS:
        assert res[0][k] == want[k]
