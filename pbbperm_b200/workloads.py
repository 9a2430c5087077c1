"""Batched and served solving workloads (bench.py --workload batch|serve).

batch: the batched configuration -- `count` instances of uneven size
(pbbperm_b200.instances.batch_instance, seeds 100, 101, ...), weak then Johnson
bound, initial bound NEH computed on the device (PBB_UB_NEH: inside the timed
solve, on both sides), all solved to optimality through one resident pool,
against solving the same instances one at a time with the single-instance
engine on the same GPU.  Every result carries an optimal schedule (a leaf's,
or NEH's when nothing improves on it), re-verified here.

serve: a Poisson request stream (instances.serving_instance, arrivals from
instances.poisson_arrivals) served by the pool with continuous batching
(requests are admitted between windows as slots and explorer memory free up),
latency = completion - arrival, against serving the same stream one request
at a time with the single-instance engine.
"""
import statistics
import time

import numpy as np

import pbbperm_b200 as pb
from pbbperm_b200.instances import batch_instance, serving_instance, poisson_arrivals


def makespan(p, perm):
    """Completion time of the last job on the last machine (plain recurrence)."""
    m, n = p.shape
    c = np.zeros(m, dtype=np.int64)
    for j in perm:
        c[0] += p[0, j]
        for k in range(1, m):
            c[k] = max(c[k - 1], c[k]) + p[k, j]
    return int(c[-1])


SEARCH = pb.Config(boundingMode=2, adaptiveBranchingMode=3)


def verified(p, r):
    """The result holds a schedule whose makespan is its cost."""
    return bool(r["has_perm"]) and makespan(p, r["perm"]) == r["cost"]


def solo_solve(p, ub=pb.UB_NEH, nb_ivms=16384, device=0):
    with pb.Engine(p, pb.Config(boundingMode=2, adaptiveBranchingMode=3, nbIVMs=nb_ivms, device=device)) as e:
        return e.solve(ub=ub)


def run_batch(count=512, pool_config=None, solo_sample=None, device=0):
    insts = [batch_instance(100 + i) for i in range(count)]
    ubs = [pb.UB_NEH] * count
    pc = pool_config or pb.PoolConfig(max_jobs=20, max_machines=20, window_s=0.02, device=device)
    t0 = time.perf_counter()
    res = pb.batch_solve(insts, ubs=ubs, config=SEARCH, pool_config=pc)
    t_batch = time.perf_counter() - t0
    ok = all(verified(p, r) for p, r in zip(insts, res))
    idx = list(range(count)) if not solo_sample else list(range(0, count, max(1, count // solo_sample)))
    t0 = time.perf_counter()
    solo = {i: solo_solve(insts[i], ubs[i], device=device) for i in idx}
    t_solo = time.perf_counter() - t0
    same = all(solo[i]["cost"] == res[i]["cost"] for i in idx)
    return dict(instances=count, batch_seconds=t_batch, batch_inst_per_s=count / t_batch,
                solo_instances=len(idx), solo_seconds=t_solo, solo_inst_per_s=len(idx) / t_solo,
                speedup=(count / t_batch) / (len(idx) / t_solo), all_verified=ok, same_optima_as_solo=same,
                nodes=int(sum(r["decomposed"] for r in res)),
                pool={k: getattr(pc, k) for k in ("warps_per_cta", "tail_warps", "core_warps", "split_depth", "share_after",
                                                  "explorers_per_instance", "window_s")})


def serve_stream(rate, count, seed=7, pool_config=None, device=0, max_resident=0):
    """Serve `count` requests of the Poisson stream at `rate` through one pool
    (continuous batching: arrivals join between windows as slots free up);
    latency = completion - arrival.  max_resident = 1 serves the same stream
    one request at a time through the same pool (the one-at-a-time side)."""
    arr = poisson_arrivals(seed, rate, count)
    insts = [serving_instance(10000 + i) for i in range(count)]
    ubs = [pb.UB_NEH] * count
    pc = pool_config or pb.PoolConfig(max_jobs=22, max_machines=20, window_s=0.002, device=device)
    if max_resident:
        pc = pb.PoolConfig(**{**vars(pc), "max_resident": max_resident})
    lat = {}
    with pb.Pool(pc) as pool:
        start = time.perf_counter()
        nxt = 0
        while len(lat) < count:
            now = time.perf_counter() - start
            while nxt < count and arr[nxt] <= now:
                pool.submit(insts[nxt], tag=nxt, ub=ubs[nxt], config=SEARCH)
                nxt += 1
            res, q = pool.step()
            done_t = time.perf_counter() - start
            for r in pool.poll():
                lat[r["tag"]] = (done_t - arr[r["tag"]], r)
            if res == 0 and q == 0 and nxt < count:
                # idle: wait for the next arrival
                wait = arr[nxt] - (time.perf_counter() - start)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
        span = time.perf_counter() - start - arr[0]
    lats = sorted(v[0] for v in lat.values())
    ok = all(verified(insts[t], r) for t, (_, r) in lat.items())
    return dict(rate=rate, requests=count, throughput=count / span, p50_ms=1e3 * lats[len(lats) // 2],
                p99_ms=1e3 * lats[min(len(lats) - 1, int(0.99 * len(lats)))], all_verified=ok,
                costs={t: r["cost"] for t, (_, r) in lat.items()})


def alone_service(count, device=0):
    """Solve the first `count` requests of the stream one at a time with the
    single-instance engine; returns their service times (s) and optima.  The
    request sequence does not depend on the rate, so one measurement serves
    every rate of a sweep."""
    insts = [serving_instance(10000 + i) for i in range(count)]
    ubs = [pb.UB_NEH] * count
    service, costs = [], {}
    for i in range(count):
        t0 = time.perf_counter()
        r = solo_solve(insts[i], ubs[i], device=device)
        service.append(time.perf_counter() - t0)
        costs[i] = r["cost"]
    return service, costs


def alone_fifo(rate, service, seed=7):
    """Latencies of the stream at `rate` served one request at a time (FIFO)
    with the measured service times: service starts at max(arrival, previous
    end)."""
    count = len(service)
    arr = poisson_arrivals(seed, rate, count)
    t_free = 0.0
    lats = []
    for i in range(count):
        begin = max(arr[i], t_free)
        t_free = begin + service[i]
        lats.append(t_free - arr[i])
    lats_s = sorted(lats)
    return dict(rate=rate, requests=count, throughput=count / (t_free - arr[0]),
                capacity=count / sum(service), mean_service_ms=1e3 * statistics.mean(service),
                p50_ms=1e3 * lats_s[len(lats_s) // 2], p99_ms=1e3 * lats_s[min(count - 1, int(0.99 * count))])
