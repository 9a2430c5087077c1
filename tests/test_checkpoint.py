"""Checkpoint files in the reference's works::save form
(distributed/src/works.cpp:172-190): the factoradic <-> decimal index
conversion (fact_work::VectToBigint / BigintToVect,
distributed/src/fact_work.cpp:49-87) on the CPU against Python integers, and
on the GPU a search saved between windows and resumed in a new engine."""
import math

import numpy as np
import pytest

from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance


def py_index(d):
    n = len(d)
    return sum(int(d[i]) * math.factorial(n - 1 - i) for i in range(n))


@pytest.mark.parametrize("n", [1, 2, 5, 13, 20, 33, 50, 64])
def test_fact_decimal_roundtrip_against_python_integers(n):
    rng = np.random.default_rng(n)
    cases = [np.zeros(n, np.int32), np.array([n - 1 - i for i in range(n)], np.int32)]
    cases += [np.array([rng.integers(0, n - i) for i in range(n)], np.int32) for _ in range(50)]
    for d in cases:
        s = pb.fact_to_decimal(d)
        assert int(s) == py_index(d)
        assert (pb.decimal_to_fact(n, s) == d).all()
    # the whole space ends at n! - 1
    assert int(pb.fact_to_decimal(np.array([n - 1 - i for i in range(n)], np.int32))) == math.factorial(n) - 1


def test_fact_decimal_rejects_bad_input():
    with pytest.raises(pb.PbbError):
        pb.fact_to_decimal(np.array([3, 0, 0], np.int32))        # digit 0 must be < 3
    with pytest.raises(pb.PbbError):
        pb.decimal_to_fact(4, str(math.factorial(4)))            # not below 4!
    with pytest.raises(pb.PbbError):
        pb.decimal_to_fact(4, "12a")


def parse_checkpoint(path):
    tok = open(path).read().split()
    n = int(tok[0])
    i = 2 + n
    root = [int(x) for x in tok[2:i]]
    simple = int(tok[i]); i += 1
    assert int(tok[i]) == n
    best_cost = int(tok[i + 1])
    best = [int(x) for x in tok[i + 2:i + 2 + n]]
    i += 2 + n
    works = int(tok[i]); i += 1
    ivs = []
    for _ in range(works):
        nb = int(tok[i + 4]); i += 5
        for _ in range(nb):
            ivs.append((int(tok[i]), int(tok[i + 1]), int(tok[i + 2]))); i += 3
        i += 1
    assert i == len(tok)
    return dict(n=n, root=root, simple=simple, best_cost=best_cost, best=best, intervals=ivs)


@pytest.mark.gpu
def test_checkpoint_file_resumes_to_the_optimum(tmp_path):
    p = synthetic_instance(24, 13, 20)
    O = Oracle(p)
    opt = 1803
    path = str(tmp_path / "bab.save")
    with pb.Engine(p, pb.Config(boundingMode=2, nbIVMs=2048)) as e:
        e.start(ub=opt + 1)
        done = e.explore(0.002)
        assert not done
        mid = e.result()
        e.save_checkpoint(path)
    ck = parse_checkpoint(path)
    assert ck["n"] == 13 and ck["simple"] == mid["simple_bounds"] and ck["best_cost"] == mid["cost"]
    assert len(ck["intervals"]) > 0
    for _, a, b in ck["intervals"]:
        assert 0 <= a <= b < math.factorial(13)
    with pb.Engine(p, pb.Config(boundingMode=2, nbIVMs=2048)) as e:
        assert e.load_checkpoint(path) == mid["simple_bounds"]
        while not e.explore(1.0):
            pass
        got = e.result()
    assert got["complete"] and got["has_perm"] and got["cost"] == opt
    assert O.eval(got["perm"]) == opt
