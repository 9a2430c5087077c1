"""Autotuner of the resident pool's shape for a batch of instances.

Times pbb_batch_solve on a calibration sample (every k-th instance of the
batch, same bounds) for each candidate block shape (warps per CTA) and explorers
per instance, and returns the fastest PoolConfig with the
timings of all candidates.
"""
import itertools
import time

import pbbperm_b200 as pb

CANDIDATES = {
    "warps_per_cta": (4, 8, 16),
    # 0: one explorer per warp of the grid, so that an instance left alone at
    # the end of a batch can still use the whole GPU (a calibration sample
    # does not show that tail)
    "explorers_per_instance": (0,),
}


def tune_pool(instances, ubs, search, max_jobs, max_machines, sample=48, window_s=0.01, device=0, repeats=1):
    step = max(1, len(instances) // sample)
    cal = instances[::step][:sample]
    cal_ub = ubs[::step][:sample]
    trials = []
    best = None
    for w, e in itertools.product(CANDIDATES["warps_per_cta"], CANDIDATES["explorers_per_instance"]):
        pc = pb.PoolConfig(max_jobs=max_jobs, max_machines=max_machines, warps_per_cta=w, explorers_per_instance=e,
                           window_s=window_s, device=device)
        t = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            pb.batch_solve(cal, ubs=cal_ub, config=search, pool_config=pc)
            t = min(t, time.perf_counter() - t0)
        trials.append(dict(warps_per_cta=w, explorers_per_instance=e, seconds=round(t, 4)))
        if best is None or t < best[0]:
            best = (t, pc)
    return best[1], trials
