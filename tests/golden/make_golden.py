#!/usr/bin/env python3
"""Generate the golden fixtures of tests/golden/ from the reference itself.

Requires the reference checker built by oracle/build_ref.py (oracle/_ref/:
the reference's bounds library behind oracle/ref_shim.cpp, and its multicore
B&B `bb` / `bbJ`).  Instances come from the project's seeded generator
(pbbperm_b200/instances.py); no benchmark suite data is written.

  bounds_golden.json  per instance: p, sampled nodes (schedule, limit1,
                      limit2) and the reference's answers -- weak children
                      LBs (boundChildren), Johnson children LBs (bornes_calculer
                      on each child), weak and Johnson node LBs, makespan.
  search_golden.json  reference multicore B&B runs with UB = optimum:
                      TOTdecomposed / TOTjohnson LBs / TOTsimple LBs / TOTleaves
                      per (instance, boundingMode, adaptiveBranchingMode, findAll).
  sorted_golden.json  reference B&B runs on ONE thread from UB = +inf with
                      sortedDFS 0 and 1: the exploration order decides when the
                      bound improves, so the counters pin the order of the children.

Usage: python tests/golden/make_golden.py [--big] [--big-only] [--sorted-only] [--early-stop-only]
       [--priorities-only]
(--big adds the 20x20 seed-1 instance of the second configuration, several
CPU-minutes of reference time; --big-only runs just that case and replaces the
`big` entry of search_golden.json, keeping the other runs; --early-stop-only
replaces the earlyStopJohnson = true runs of both search fixtures;
--priorities-only replaces the sortedDFS 2-4 runs of sorted_golden.json)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import Oracle, Reference, run_reference_bb  # noqa: E402
from pbbperm_b200.instances import synthetic_instance  # noqa: E402

INF = 2**31 - 1

BOUND_CASES = [(8, 4, 101), (12, 10, 102), (20, 5, 0), (20, 20, 1), (33, 7, 103), (50, 20, 2), (64, 12, 104),
               (10, 32, 105), (30, 2, 106)]
NODES_PER_CASE = 40

SEARCH_CASES = [(10, 5, 21), (12, 10, 22), (14, 5, 23), (13, 20, 24), (16, 8, 25), (20, 5, 0), (11, 3, 26),
                (9, 12, 27), (15, 6, 28), (35, 10, 45)]
TINY_CASES = [(8, 4, 29), (9, 6, 30), (7, 10, 31)]
SORTED_CASES = [(9, 5, 41), (10, 5, 42), (11, 8, 43), (10, 10, 44)]
SORTED_MODES = [(0, 3), (2, 3), (2, 1), (1, 2), (2, -3)]


def child_strong(R, sched, l1, l2, front):
    n = len(sched)
    out = np.zeros(n, np.int32)
    L1 = l1 + (1 if front else 0)
    L2 = l2 - (0 if front else 1)
    fill = L1 if front else L2
    for i in range(l1 + 1, l2):
        s = sched.copy()
        s[fill], s[i] = s[i], s[fill]
        out[sched[i]] = R.strong_node(s, L1, L2)
    return out


def make_bounds():
    rng = np.random.default_rng(2024)
    cases = []
    for n, m, seed in BOUND_CASES:
        p = synthetic_instance(seed, n, m)
        R = Reference(p)
        O = Oracle(p)
        nodes = []
        for t in range(NODES_PER_CASE):
            sched = rng.permutation(n).astype(np.int32)
            if t == 0:
                nf, nb = 0, 0
            elif t == 1:
                nf, nb = n - 2, 0
            elif t == 2:
                nf, nb = 0, n - 3
            elif t == 3:
                nf, nb = n // 2, n - n // 2 - 1
            else:
                nf = int(rng.integers(0, n - 1))
                nb = int(rng.integers(0, n - nf))
            l1, l2 = nf - 1, n - nb
            cb, ce, _, _ = R.weak_children(sched, l1, l2)
            rec = dict(sched=sched.tolist(), l1=l1, l2=l2,
                       weak_begin=cb.tolist(), weak_end=ce.tolist(),
                       strong_begin=child_strong(R, sched, l1, l2, True).tolist(),
                       strong_end=child_strong(R, sched, l1, l2, False).tolist(),
                       node_weak=int(R.weak_node(sched, l1, l2)), node_strong=int(R.strong_node(sched, l1, l2)),
                       makespan=int(R.eval(sched)))
            # the oracle must agree before anything is written
            ocb, oce, _, _ = O.weak_children(sched, l1, l2)
            assert (ocb == cb).all() and (oce == ce).all()
            assert (O.strong_children(sched, l1, l2, True) == np.array(rec["strong_begin"])).all()
            assert (O.strong_children(sched, l1, l2, False) == np.array(rec["strong_end"])).all()
            assert O.strong_node(sched, l1, l2) == rec["node_strong"]
            nodes.append(rec)
        johnson = [R.johnson_row(s).tolist() for s in range(m * (m - 1) // 2)]
        cases.append(dict(n=n, m=m, seed=seed, p=p.tolist(), nodes=nodes, johnson=johnson))
    with open(os.path.join(HERE, "bounds_golden.json"), "w") as f:
        json.dump(dict(source="reference bounds library (oracle/_ref/libref_bounds.so)", cases=cases), f)


def make_search(big=False):
    runs = []
    main = [(0, 3, False), (1, 3, False), (2, 3, False), (2, 1, False), (2, 2, False), (0, 1, False),
            (0, 2, False), (2, 3, True), (0, 3, True)]
    # fixed-side rules: with the weak bound the reference never fills the
    # back-side costs for them (bounds/src/bound_fsp_weak.cpp:209-216), so the
    # back side is never pruned -- tiny instances only
    fixed = [(2, -1, False), (0, -1, False), (0, -2, False), (2, -2, False), (2, -3, False), (1, -2, False)]
    cases = [(c, main) for c in SEARCH_CASES] + [(c, fixed) for c in TINY_CASES]
    cases.append(((50, 20, 2), [(0, 3, False), (2, 3, False)]))
    for (n, m, seed), combos in cases:
        p = synthetic_instance(seed, n, m)
        O = Oracle(p)
        if (n, m, seed) == (50, 20, 2):
            opt, ub = None, 3780          # below the optimum: deterministic, nothing found
        else:
            opt = O.solve(INF, bound_mode=2)["best"]
            ub = opt
        for bm, br, fa in combos:
            try:
                r = run_reference_bb(p, ub=ub, bound_mode=bm, branch_mode=br, threads=8, johnson=(bm != 0),
                                     find_all=fa, timeout=300)
            except Exception as exc:  # a reference run that does not finish in time is left out
                print("skip", n, m, seed, bm, br, fa, exc)
                continue
            o = O.solve(ub, bound_mode=bm, branch_mode=br, find_all=fa, node_limit=5000000)
            rec = dict(n=n, m=m, seed=seed, opt=opt, ub=ub, bounding_mode=bm, branching_mode=br, find_all=fa,
                       decomposed=r["decomposed"], johnson_bounds=r["johnson_bounds"],
                       simple_bounds=r["simple_bounds"], leaves=r["leaves"])
            if o["complete"]:
                for k in ("decomposed", "johnson_bounds", "simple_bounds", "leaves"):
                    assert o[k] == rec[k], (n, m, seed, bm, br, fa, k, o[k], rec[k])
            runs.append(rec)
            print("run", n, m, seed, bm, br, fa, rec["decomposed"], flush=True)
    # UB = +inf with the weak bound (20x5, seed 0): only the optimum is deterministic
    p = synthetic_instance(0, 20, 5)
    r = run_reference_bb(p, ub=None, bound_mode=0, branch_mode=3, threads=8, johnson=False)
    runs.append(dict(n=20, m=5, seed=0, ub=None, bounding_mode=0, branching_mode=3, find_all=False,
                     opt=r["best"], perm=r["perm"]))
    if big:
        runs.append(big_run())
    else:
        old = os.path.join(HERE, "search_golden.json")
        if os.path.exists(old):
            with open(old) as f:
                runs += [r for r in json.load(f)["runs"] if r.get("big")]
    with open(os.path.join(HERE, "search_golden.json"), "w") as f:
        json.dump(dict(source="reference multicore B&B (oracle/_ref/bb, bbJ), 8 threads", runs=runs), f, indent=0)


def big_run():
    """The second configuration: 20 jobs x 20 machines (seed 1), weak then
    Johnson bound, MinMin, UB = its optimum 2352 (found by the reference from
    UB = +inf), 8 reference threads: the node counters are deterministic."""
    p = synthetic_instance(1, 20, 20)
    opt = 2352
    r = run_reference_bb(p, ub=opt, bound_mode=2, branch_mode=3, threads=8, johnson=True, timeout=20000)
    print("big", r, flush=True)
    return dict(n=20, m=20, seed=1, opt=opt, ub=opt, bounding_mode=2, branching_mode=3, find_all=False,
                decomposed=r["decomposed"], johnson_bounds=r["johnson_bounds"],
                simple_bounds=r["simple_bounds"], leaves=r["leaves"], big=True)


EARLY_STOP_MODES = [(2, 3), (2, 1), (2, 2), (1, 3), (1, 2)]


def make_early_stop():
    """Reference runs with earlyStopJohnson = true (its default): at UB =
    optimum on 8 threads (deterministic counters), and on ONE thread from
    UB = +inf with sortedDFS 0 and 1.  Appended to search_golden.json /
    sorted_golden.json with early_stop = true, replacing earlier such runs.
    boundingMode 1 with MaxSum is left out: there the reference's counters
    depend on each thread's machine-pair success history."""
    path = os.path.join(HERE, "search_golden.json")
    with open(path) as f:
        g = json.load(f)
    runs = [r for r in g["runs"] if not r.get("early_stop")]
    for n, m, seed in SEARCH_CASES[:6]:
        p = synthetic_instance(seed, n, m)
        opt = Oracle(p).solve(INF, bound_mode=2)["best"]
        for bm, br in EARLY_STOP_MODES:
            r = run_reference_bb(p, ub=opt, bound_mode=bm, branch_mode=br, threads=8, johnson=True,
                                 early_stop=True, timeout=600)
            runs.append(dict(n=n, m=m, seed=seed, opt=opt, ub=opt, bounding_mode=bm, branching_mode=br,
                             find_all=False, early_stop=True, decomposed=r["decomposed"],
                             johnson_bounds=r["johnson_bounds"], simple_bounds=r["simple_bounds"],
                             leaves=r["leaves"]))
            print("early-stop run", n, m, seed, bm, br, r["decomposed"], flush=True)
    g["runs"] = runs
    with open(path, "w") as f:
        json.dump(g, f, indent=0)
    path = os.path.join(HERE, "sorted_golden.json")
    with open(path) as f:
        g = json.load(f)
    runs = [r for r in g["runs"] if not r.get("early_stop")]
    for n, m, seed in SORTED_CASES[:2]:
        p = synthetic_instance(seed, n, m)
        for bm, br in [(2, 3), (1, 2)]:
            for sd in (0, 1):
                r = run_reference_bb(p, ub=None, bound_mode=bm, branch_mode=br, threads=1, johnson=True,
                                     sorted_dfs=sd, early_stop=True, timeout=600)
                runs.append(dict(n=n, m=m, seed=seed, p=p.tolist(), bounding_mode=bm, branching_mode=br,
                                 sorted_dfs=sd, early_stop=True, best=r["best"], decomposed=r["decomposed"],
                                 johnson_bounds=r["johnson_bounds"], simple_bounds=r["simple_bounds"],
                                 leaves=r["leaves"]))
    g["runs"] = runs
    with open(path, "w") as f:
        json.dump(g, f, indent=0)


PRIORITY_MODES = [(0, 3), (2, 3), (2, 1), (1, 2), (2, -3)]


def make_priorities():
    """sortedDFS 2-4 with sortingCriterion 1-3 on ONE reference thread from
    UB = +inf: rows sorted by (first cost, priority) or by the priority
    (ivm_bound.cpp:338-370, priorities :506-544).  Appended to
    sorted_golden.json with their sorting_criterion, replacing earlier such
    runs.  Left out: criterion 3 with boundingMode 1 (the reference reads an
    unset Johnson idle time for children with one free job) and criterion 4
    (completeSchedule writes past the node's free block)."""
    path = os.path.join(HERE, "sorted_golden.json")
    with open(path) as f:
        g = json.load(f)
    runs = [r for r in g["runs"] if r["sorted_dfs"] <= 1]
    for n, m, seed in SORTED_CASES:
        p = synthetic_instance(seed, n, m)
        for bm, br in PRIORITY_MODES:
            for sd in (2, 3, 4):
                for crit in (1, 2, 3):
                    if bm == 1 and crit == 3:
                        continue
                    r = run_reference_bb(p, ub=None, bound_mode=bm, branch_mode=br, threads=1, johnson=(bm != 0),
                                         sorted_dfs=sd, sorting_criterion=crit, timeout=600)
                    runs.append(dict(n=n, m=m, seed=seed, p=p.tolist(), bounding_mode=bm, branching_mode=br,
                                     sorted_dfs=sd, sorting_criterion=crit, best=r["best"],
                                     decomposed=r["decomposed"], johnson_bounds=r["johnson_bounds"],
                                     simple_bounds=r["simple_bounds"], leaves=r["leaves"]))
    g["runs"] = runs
    with open(path, "w") as f:
        json.dump(g, f, indent=0)


def make_big_only():
    path = os.path.join(HERE, "search_golden.json")
    with open(path) as f:
        g = json.load(f)
    g["runs"] = [r for r in g["runs"] if not r.get("big")] + [big_run()]
    with open(path, "w") as f:
        json.dump(g, f, indent=0)


def make_sorted():
    runs = []
    for n, m, seed in SORTED_CASES:
        p = synthetic_instance(seed, n, m)
        for bm, br in SORTED_MODES:
            for sd in (0, 1):
                r = run_reference_bb(p, ub=None, bound_mode=bm, branch_mode=br, threads=1, johnson=(bm != 0),
                                     sorted_dfs=sd, timeout=600)
                runs.append(dict(n=n, m=m, seed=seed, p=p.tolist(), bounding_mode=bm, branching_mode=br,
                                 sorted_dfs=sd, best=r["best"], decomposed=r["decomposed"],
                                 johnson_bounds=r["johnson_bounds"], simple_bounds=r["simple_bounds"],
                                 leaves=r["leaves"]))
    with open(os.path.join(HERE, "sorted_golden.json"), "w") as f:
        json.dump(dict(source="reference multicore B&B (oracle/_ref/bb, bbJ), 1 thread, UB = +inf", runs=runs),
                  f, indent=0)


if __name__ == "__main__":
    if not oracle.reference_available():
        sys.exit("build the reference checker first: python oracle/build_ref.py")
    if "--priorities-only" in sys.argv:
        make_priorities()
        print("sortedDFS 2-4 runs written")
        sys.exit(0)
    if "--early-stop-only" in sys.argv:
        make_early_stop()
        print("early-stop runs written")
        sys.exit(0)
    if "--big-only" in sys.argv:
        make_big_only()
        print("search_golden.json: big run replaced")
        sys.exit(0)
    if "--sorted-only" not in sys.argv:
        if "--search-only" not in sys.argv:
            make_bounds()
        make_search(big="--big" in sys.argv)
    make_sorted()
    print("golden fixtures written to", HERE)
