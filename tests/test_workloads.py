"""Host logic of the batched and served workloads (no GPU): the instance
generators' shapes and determinism, the Poisson stream, the makespan used to
re-verify returned permutations, the one-at-a-time FIFO latency model, and the
factoradic slices the ranks of a multi-GPU run take."""
import numpy as np

import bench
from oracle import Oracle
from pbbperm_b200 import workloads
from pbbperm_b200.instances import batch_instance, poisson_arrivals, serving_instance, synthetic_instance


def test_batch_instances_have_the_configured_shapes_and_repeat():
    shapes = set()
    for seed in range(100, 160):
        p = batch_instance(seed)
        m, n = p.shape
        assert 12 <= n <= 20 and m in (5, 10, 20)
        assert p.dtype == np.int32 and p.min() >= 1 and p.max() <= 99
        assert np.array_equal(p, batch_instance(seed))
        shapes.add((n, m))
    assert len({m for _, m in shapes}) == 3           # every machine count occurs


def test_serving_instances_have_the_configured_shapes():
    for seed in range(10000, 10040):
        p = serving_instance(seed)
        m, n = p.shape
        assert 10 <= n <= 22 and 5 <= m <= 20
        assert p.min() >= 1 and p.max() <= 99


def test_poisson_stream_is_increasing_with_the_right_mean_gap():
    a = poisson_arrivals(7, 100.0, 20000)
    assert np.all(np.diff(a) > 0)
    assert abs(np.mean(np.diff(a)) - 0.01) < 0.0005     # 1/rate within 5 %
    assert np.array_equal(a, poisson_arrivals(7, 100.0, 20000))


def test_makespan_matches_the_oracle_evaluation():
    rng = np.random.default_rng(3)
    for seed, n, m in [(1, 20, 20), (4, 13, 7), (9, 30, 5)]:
        p = synthetic_instance(seed, n, m)
        O = Oracle(p)
        for _ in range(5):
            perm = rng.permutation(n)
            assert workloads.makespan(p, perm) == O.eval(perm)


def test_fifo_latencies_of_one_at_a_time_serving():
    service = [1.0, 0.5, 2.0]
    r = workloads.alone_fifo(1e6, service)            # everything arrives at once
    assert abs(r["capacity"] - 3 / 3.5) < 1e-12
    assert r["p99_ms"] > r["p50_ms"] > 0
    slow = workloads.alone_fifo(1e-3, service)        # arrivals far apart: no queueing
    assert abs(slow["p99_ms"] - 2000.0) < 1e-6


def test_rank_slices_cover_the_first_level_once():
    for n in (13, 50):
        for world in (1, 2, 3, 8):
            if world == 1:
                assert bench.rank_slice(n, 0, world) is None
                continue
            cells = []
            for r in range(world):
                sl = bench.rank_slice(n, r, world)
                if sl is None:
                    continue
                pos, end = sl
                assert len(pos) == n and len(end) == n
                assert all(0 <= pos[i] < n - i and 0 <= end[i] < n - i for i in range(n))
                cells.extend(range(pos[0], end[0] + 1))
            assert sorted(cells) == list(range(n))
