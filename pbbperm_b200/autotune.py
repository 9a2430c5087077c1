"""Autotuner of the resident pool's shape for a batch of instances.

Times pbb_batch_solve on a calibration sample of the batch and searches, one
dimension at a time from the defaults (coordinate descent, each dimension's
best value kept before the next is tried):

  warps_per_cta           block shape of the bulk of the batch
  tail_warps              block shape once few instances remain (0 = 20 warps, -1 = none)
  core_warps              warps per CTA that always ask for work (steal threshold)
  split_depth             no split deeper than n - split_depth (steal threshold)
  share_after             nodes an explorer decomposes before it offers work again (steal threshold)
  explorers_per_instance  explorers of each resident instance (0 = one per warp of the widest grid)
  window_s                device time of a window while instances wait (admission granularity)

The sample is every k-th instance plus the largest ones (jobs x machines):
a batch ends with its heaviest searches, which a uniform sample misses.
Returns the fastest PoolConfig and the timings of every trial.
"""
import time

import pbbperm_b200 as pb

CANDIDATES = [
    ("warps_per_cta", (8, 4, 16)),
    ("tail_warps", (0, -1)),
    ("core_warps", (8, 4)),
    ("split_depth", (10, 6, 14)),
    ("share_after", (64, 16, 256)),
    ("explorers_per_instance", (0, 1024)),
    ("window_s", (0.01, 0.004, 0.02)),
]


def calibration_sample(instances, ubs, size=32, largest=2):
    order = sorted(range(len(instances)), key=lambda i: (-instances[i].size, -instances[i].shape[1], i))
    top = order[:largest]
    step = max(1, len(instances) // size)
    idx = sorted(set(top) | set(range(0, len(instances), step)))
    return [instances[i] for i in idx], [ubs[i] for i in idx]


def tune_pool(instances, ubs, search, max_jobs, max_machines, sample=32, device=0, repeats=1, largest=2):
    cal, cal_ub = calibration_sample(instances, ubs, sample, largest)
    current = {k: v[0] for k, v in CANDIDATES}
    trials = []
    cache = {}

    def timed(cfg):
        key = tuple(sorted(cfg.items()))
        if key in cache:
            return cache[key]
        pc = pb.PoolConfig(max_jobs=max_jobs, max_machines=max_machines, device=device, **cfg)
        t = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            pb.batch_solve(cal, ubs=cal_ub, config=search, pool_config=pc)
            t = min(t, time.perf_counter() - t0)
        cache[key] = t
        trials.append(dict(cfg, seconds=round(t, 4)))
        return t

    best_t = timed(current)
    for name, values in CANDIDATES:
        for v in values[1:]:
            trial = dict(current, **{name: v})
            t = timed(trial)
            if t < best_t:
                best_t, current = t, trial
    pc = pb.PoolConfig(max_jobs=max_jobs, max_machines=max_machines, device=device, **current)
    return pc, trials
