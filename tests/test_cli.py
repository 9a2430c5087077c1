"""The drop-in command line `pbbperm_b200/bb -z p=fsp,i=<instance>[,o]`
(gpu/src/main.cpp:12-77 of the reference): it reads ./gpuconfig.ini and the
reference's parameter files from the working directory and prints the
reference's statistics keys, which oracle.parse_bb_output reads for both
programs.  Errors in the arguments or the files are caught before any GPU
work (CPU tests); the searches themselves run on the GPU."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from oracle import Oracle, parse_bb_output, write_vrf
from pbbperm_b200.instances import synthetic_instance

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BB = os.path.join(ROOT, "pbbperm_b200", "bb")
KEYS = ("decomposed", "johnson_bounds", "simple_bounds", "leaves")

needs_bb = pytest.mark.skipif(not os.path.exists(BB), reason="command line not built")


def write_ini(d, instance, ub_mode, nb_ivms=1024, sorted_dfs=0, extra=""):
    with open(os.path.join(d, "gpuconfig.ini"), "w") as f:
        f.write("[problem]\nproblem = flowshop\ninstance = %s\n" % instance)
        f.write("[initial]\nub = %d\nsol = 0\n" % ub_mode)
        f.write("[bb]\nboundingMode = 2\nadaptiveBranchingMode = 3\nJohnsonMode = 0\n")
        f.write("earlyStopJohnson = false\nfindAll = false\n")
        if sorted_dfs is not None:
            f.write("sortedDFS = %d\n" % sorted_dfs)
        f.write("[gpu]\nnbIVMs = %d\n" % nb_ivms)
        f.write(extra)


def run_bb(d, args):
    return subprocess.run([BB] + args, cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                          timeout=600)


@needs_bb
def test_missing_instance_file_is_an_error(tmp_path):
    write_ini(tmp_path, "VNOPE", 0)
    r = run_bb(tmp_path, ["-z", "p=fsp,i=VNOPE,o"])
    assert r.returncode != 0
    assert "vrf_parameters/VNOPE_Gap.txt" in r.stdout


@needs_bb
def test_other_problems_are_refused(tmp_path):
    write_ini(tmp_path, "VX", 0)
    r = run_bb(tmp_path, ["-z", "p=nqueens,i=VX"])
    assert r.returncode != 0
    assert "flow-shop" in r.stdout


@pytest.mark.gpu
@needs_bb
def test_vrf_instance_at_the_optimum_counts_like_the_oracle(tmp_path):
    """`,o` takes the best known value from instancesVRF.data as the UB: the
    counters the command line prints equal the oracle's at that UB."""
    p = synthetic_instance(24, 13, 20)
    write_vrf(str(tmp_path), "VCLI13x20", p, ub=1803)
    write_ini(tmp_path, "VCLI13x20", 0)
    r = run_bb(tmp_path, ["-z", "p=fsp,i=VCLI13x20,o"])
    assert r.returncode == 0, r.stdout
    got = parse_bb_output(r.stdout)
    want = Oracle(p).solve(1803, bound_mode=2)
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.gpu
@needs_bb
def test_default_sorted_dfs_from_infinity_on_one_explorer(tmp_path, sorted_golden):
    """An ini without sortedDFS means sortedDFS = 1 in the reference; from
    UB = +inf on one explorer the printed counters and optimum equal the
    reference's single-thread run."""
    run = next(r for r in sorted_golden["runs"] if r["seed"] == 43 and r["bounding_mode"] == 2
               and r["branching_mode"] == 3 and r["sorted_dfs"] == 1)
    p = np.array(run["p"], np.int32)
    write_vrf(str(tmp_path), "VSORT", p, ub=None)
    write_ini(tmp_path, "VSORT", 3, nb_ivms=1, sorted_dfs=None)
    r = run_bb(tmp_path, ["-z", "p=fsp,i=VSORT"])
    assert r.returncode == 0, r.stdout
    got = parse_bb_output(r.stdout)
    for k in KEYS:
        assert got[k] == run[k], (k, got[k], run[k])
    assert got.get("best") == run["best"]
