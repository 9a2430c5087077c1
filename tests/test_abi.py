"""The C ABI library without a GPU: symbols, argument checks, host-only code."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance, read_vrf, write_vrf

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            names.update(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(pbb_\w+)\s*\(", text, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = pb.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), name


def test_invalid_instances_rejected_before_cuda():
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(np.ones((2, 100), np.int32))
    assert e.value.code == pb.PBB_E_INVAL
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(np.ones((40, 10), np.int32))
    assert e.value.code == pb.PBB_E_INVAL
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(np.full((3, 10), 70000, np.int32))
    assert e.value.code == pb.PBB_E_INVAL


def test_unsupported_options_rejected():
    p = synthetic_instance(0, 10, 4)
    with pytest.raises(pb.PbbError) as e:
        # early Johnson exit where pruned children's values choose the side
        pb.Engine(p, pb.Config(earlyStopJohnson=True, boundingMode=1, adaptiveBranchingMode=1))
    assert e.value.code == pb.PBB_E_UNSUPPORTED
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(p, pb.Config(sortedDFS=2, sortingCriterion=4))    # undefined in the reference
    assert e.value.code == pb.PBB_E_UNSUPPORTED
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(p, pb.Config(sortedDFS=3, sortingCriterion=3, boundingMode=1))
    assert e.value.code == pb.PBB_E_UNSUPPORTED
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(p, pb.Config(sortedDFS=5))
    assert e.value.code == pb.PBB_E_INVAL
    with pytest.raises(pb.PbbError) as e:
        pb.Engine(p, pb.Config(adaptiveBranchingMode=4))
    assert e.value.code == pb.PBB_E_INVAL


def test_bound_children_validates_nodes():
    p = synthetic_instance(0, 10, 4)
    bad = np.zeros((1, 10), np.int32)  # not a permutation
    with pytest.raises(pb.PbbError) as e:
        pb.bound_children(p, bad, [-1], [10])
    assert e.value.code == pb.PBB_E_INVAL
    good = np.arange(10, dtype=np.int32)[None]
    with pytest.raises(pb.PbbError):
        pb.bound_children(p, good, [5], [5])


def test_neh_matches_oracle():
    for seed, n, m in [(0, 20, 5), (1, 20, 20), (2, 50, 20), (9, 7, 3)]:
        p = synthetic_instance(seed, n, m)
        c, perm = pb.neh(p)
        oc, operm = oracle.Oracle(p).neh()
        assert c == oc and (perm == operm).all()


def test_vrf_roundtrip(tmp_path):
    p = synthetic_instance(3, 13, 6)
    path = str(tmp_path / "VTEST_Gap.txt")
    write_vrf(path, p)
    assert (read_vrf(path) == p).all()
