"""The C ABI library without a GPU: symbols, argument checks, host-only code."""
import ctypes
import os
import re
import subprocess

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


STRUCTS = [("pbb_instance", "_Instance"), ("pbb_config", "_Config"), ("pbb_stats", "_Stats"),
           ("pbb_result", "_Result"), ("pbb_work", "_Work"), ("pbb_pool_config", "_PoolConfig"),
           ("pbb_pool_result", "_PoolResult"), ("pbb_bound_out", "_BoundOut")]


def test_python_struct_mirrors_match_the_c_headers(tmp_path):
    """Every ctypes mirror in pbbperm_b200 has the C struct's size and each
    field's offset, as gcc lays them out from include/*.h."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pbbperm.h"', '#include "pbbperm_diag.h"',
             'int main(void) {']
    for c_name, py_name in STRUCTS:
        S = getattr(pb, py_name)
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (c_name, c_name))
        for f in S._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (c_name, f[0], c_name, f[0]))
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            a, b, v = line.split()
            got[(a, b)] = int(v)
    for c_name, py_name in STRUCTS:
        S = getattr(pb, py_name)
        assert got[(c_name, "size")] == ctypes.sizeof(S), c_name
        for f in S._fields_:
            assert got[(c_name, f[0])] == getattr(S, f[0]).offset, (c_name, f[0])
