"""Interval import and export (gpubb::initFromFac / getIntervals, the form the
reference's distributed workers exchange work in): several explorers started
at once on disjoint intervals count exactly what the oracle counts on each
interval, and a checkpoint taken between windows resumes to the end in
another engine."""
import numpy as np
import pytest

import bench
from oracle import Oracle
import pbbperm_b200 as pb
from pbbperm_b200.instances import synthetic_instance

pytestmark = pytest.mark.gpu

KEYS = ("decomposed", "johnson_bounds", "simple_bounds", "leaves")
OPT = 1803          # optimum of the 13x20 instance of seed 24


def run_to_end(e, window=1.0):
    while not e.explore(window):
        pass
    return e.result()


@pytest.mark.parametrize("ids", [None, [7, 0, 33]])
def test_init_from_fac_counts_equal_oracle_sum(ids):
    p = synthetic_instance(24, 13, 20)
    O = Oracle(p)
    slices = [bench.rank_slice(13, r, 3) for r in range(3)]
    want = {k: 0 for k in KEYS}
    for pos, end in slices:
        w = O.solve(OPT, bound_mode=2, pos=pos, end=end)
        assert not w["found"]
        for k in KEYS:
            want[k] += w[k]
    pos = np.stack([s[0] for s in slices])
    end = np.stack([s[1] for s in slices])
    with pb.Engine(p, pb.Config(nbIVMs=64, boundingMode=2)) as e:
        e.init_from_fac(OPT, pos, end, ids=ids)
        got = run_to_end(e)
    assert got["complete"] and not got["found"]
    for k in KEYS:
        assert got[k] == want[k], (k, got[k], want[k])


def test_checkpoint_between_windows_resumes_to_the_end():
    """Stop after a short window, export the intervals still held, resume them
    in a smaller engine.  The resumed explorers re-bound their start paths
    without counting them (initAtInterval), so the two counts add up to at
    most the uninterrupted count and fall short of it by at most one path of
    n nodes per resumed interval."""
    p = synthetic_instance(24, 13, 20)
    n = p.shape[1]
    full = Oracle(p).solve(OPT, bound_mode=2)
    with pb.Engine(p, pb.Config(nbIVMs=1024, boundingMode=2)) as a:
        a.start(ub=OPT)
        done = a.explore(0.0005)
        first = a.result()
        pos, end, ids = a.get_intervals()
    if done:
        pytest.skip("the search ended inside the first window")
    assert len(pos) > 0 and (ids >= 0).all() and (ids < 1024).all()
    for k in range(len(pos)):
        assert list(pos[k]) <= list(end[k])            # lexicographic interval
    with pb.Engine(p, pb.Config(nbIVMs=max(64, len(pos)), boundingMode=2)) as b:
        b.init_from_fac(OPT, pos, end)
        second = run_to_end(b)
    assert second["complete"] and not second["found"]
    total = first["decomposed"] + second["decomposed"]
    assert full["decomposed"] - n * len(pos) <= total <= full["decomposed"]


def test_interval_arguments_are_checked():
    p = synthetic_instance(24, 13, 20)
    with pb.Engine(p, pb.Config(nbIVMs=8, boundingMode=2)) as e:
        pos = np.zeros((2, 13), np.int32)
        end = np.tile(np.arange(12, -1, -1, dtype=np.int32), (2, 1))
        with pytest.raises(pb.PbbError):
            e.init_from_fac(OPT, pos, end, ids=[3, 3])          # same explorer twice
        with pytest.raises(pb.PbbError):
            e.init_from_fac(OPT, pos, end, ids=[0, 8])          # beyond nb_ivms
        bad = end.copy()
        bad[0, 0] = 13                                           # digit 0 must be < 13
        with pytest.raises(pb.PbbError):
            e.init_from_fac(OPT, pos, bad)
