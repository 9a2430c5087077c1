/*
 * pbbperm.h -- C ABI of the B200 IVM branch-and-bound engine for the
 * permutation flow-shop (makespan).  Plain pointers and sizes only; every call
 * returns a status code (PBB_OK or a negative PBB_E_*), never exits.
 *
 * Reference interfaces each entry point stands in for (jangmys/PBBPerm):
 *   pbb_engine_create   gpubb::gpubb + initialize + initializeBoundFSP + copyH2D
 *                       (gpu/include/gpubb.h:26,151,119,142; gpu/src/gpubb.cu:24-74,
 *                       83-95, 1004-1062, 917-1003), instance from instance_abstract
 *                       (bounds/include/instance_abstract.h:6-9)
 *   pbb_solve           gpubb::initFullInterval + next + getStats
 *                       (gpubb.h:36,160,168; gpubb.cu:96,273,1063; gpu/src/main.cpp:52-67)
 *                       and the statistics printed by pbab::printStats (common/src/pbab.cpp:40-74)
 *   pbb_start / pbb_explore / pbb_get_result
 *                       the same loop in resumable windows (gpubb::next(int&,int&),
 *                       gpubb.h:161; gpubb::interruptExploration gpubb.h:35;
 *                       matrix_controller::interruptExploration
 *                       multicore/src/matrix_controller.cpp:459-462)
 *   pbb_save_checkpoint / pbb_load_checkpoint
 *                       works::save / works::init_infile (distributed/src/works.cpp:61-90,172-190)
 *   pbb_start_interval / pbb_init_from_fac / pbb_get_intervals
 *                       gpubb::initAtInterval / initFromFac / getIntervals
 *                       (gpubb.h:155,171,172; gpubb.cu:1190-1310)
 *   pbb_bound_children  bound_abstract::boundChildren + bornes_calculer
 *                       (bounds/include/bound_abstract.h:15-26) for a batch of nodes
 *   pbb_bound_children_ex  the same with the idle-time priorities and couts[1]
 *   pbb_neh             fastNEH::runNEH initial upper bound (heuristic/src/fastNEH.cpp:230-243)
 *   pbb_neh_batch       the same on the device for many instances (fastNEH.cpp:100-243)
 *   pbb_ig_batch        IG::runIG iterated greedy on the device (heuristic/src/IG.cpp:341-416)
 *   pbb_engine_destroy  gpubb::~gpubb (gpubb.h:27; gpubb.cu:75)
 */
#ifndef PBBPERM_H
#define PBBPERM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PBB_OK 0
#define PBB_E_INVAL (-1)       /* bad argument or unsupported instance/config */
#define PBB_E_NOMEM (-2)       /* device allocation failed */
#define PBB_E_CUDA (-3)        /* CUDA runtime error (message in pbb_last_error) */
#define PBB_E_TIMEOUT (-4)     /* the host's wait for a window ran out (pbb_set_wait_limit) */
#define PBB_E_UNSUPPORTED (-5) /* option the engine does not implement */

#define PBB_MAX_JOBS 64
#define PBB_MAX_MACHINES 32

/* Initial bound value asking for NEH computed on the device (pbb_start,
 * pbb_solve, pbb_pool_submit, pbb_batch_solve): the search starts from the
 * NEH makespan, the reference's heuristic start ([initial] ub = 1,
 * common/src/pbab.cpp:196-200), with no host round trip. */
#define PBB_UB_NEH (-1)

/* Instance: n_jobs x n_machines processing times, row-major machine-major
 * (p[k * n_jobs + j] = time of job j on machine k), the order of the
 * reference's instance stream (bounds/src/instance_flowshop.cpp:91-101). */
typedef struct pbb_instance {
    int32_t n_jobs;
    int32_t n_machines;
    const int32_t* p;
} pbb_instance;

/* Search settings; field names follow the reference ini keys
 * (common/src/arguments.cpp:80-132). */
typedef struct pbb_config {
    int32_t bounding_mode;      /* [bb] boundingMode: 0 weak, 1 Johnson, 2 weak then Johnson */
    int32_t branching_mode;     /* [bb] adaptiveBranchingMode (CPU numbering): -3,-2,-1,1,2,3 */
    int32_t find_all;           /* [bb] findAll */
    int32_t johnson_mode;       /* [bb] JohnsonMode: 0 all pairs, 1 (k,m), 2 (k,k+1) */
    int32_t early_stop_johnson; /* [bb] earlyStopJohnson: 1 = a child's Johnson scan stops once it exceeds
                                   the incumbent (same nodes; rejected with boundingMode 1 + MaxSum) */
    int32_t sorted_dfs;         /* [bb] sortedDFS: 0 reverse the row on a side change; 1 sort it by the
                                   chosen side's bound; 2 and 4 by (bound, priority); 3 by the priority
                                   (ivm_bound.cpp:338-370) */
    int32_t nb_ivms;            /* [gpu] nbIVMs: explorers */
    int32_t device;             /* CUDA device ordinal */
    int32_t warps_per_cta;      /* 0 = largest that fits shared memory */
    int32_t ctas;               /* 0 = SMs x resident CTAs per SM */
    int32_t sorting_criterion;  /* [bb] sortingCriterion, the sibling priority of sortedDFS 2-4
                                   (ivm_bound.cpp:506-544): 1 the chosen side's bound, 2 that bound
                                   minus the other side's, 3 the weak bound's idle time (not with
                                   boundingMode 1); 4 is rejected */
    int32_t core_warps;         /* work sharing: warps per CTA that ask for work whatever the search's
                                   width; the others join once it is wide (0 = 8) */
    int32_t split_depth;        /* work sharing: no split at levels deeper than n - split_depth (0 = 10) */
    int32_t share_after;        /* work sharing: an explorer hands part of its interval to an idle one only
                                   after decomposing this many nodes since it got its interval or last
                                   gave part away (0 = 64; < 0 = at every step). Node counts do not
                                   depend on it */
} pbb_config;

typedef struct pbb_stats {
    uint64_t decomposed;        /* TOTdecomposed */
    uint64_t johnson_bounds;    /* TOTjohnson LBs */
    uint64_t simple_bounds;     /* TOTsimple LBs */
    uint64_t leaves;            /* TOTleaves */
    uint64_t steals;            /* intervals handed between explorers */
} pbb_stats;

typedef struct pbb_result {
    int32_t complete;           /* 1: the whole search space was explored */
    int32_t found;              /* 1: a leaf improved the initial bound ("Found optimal solution") */
    int32_t cost;               /* best makespan known (the initial bound if not improved) */
    int32_t n_jobs;
    int32_t perm[PBB_MAX_JOBS]; /* best permutation when found */
    pbb_stats stats;
    double device_seconds;      /* device time of the exploration kernels */
    int32_t has_perm;           /* 1: perm holds a schedule of makespan `cost` -- a leaf found it, or
                                   the search started from PBB_UB_NEH and did not improve on NEH */
    int32_t pad;
} pbb_result;

typedef struct pbb_engine pbb_engine;

void pbb_config_default(pbb_config* cfg);
const char* pbb_last_error(void);

int pbb_engine_create(const pbb_instance* inst, const pbb_config* cfg, pbb_engine** out);
int pbb_engine_destroy(pbb_engine* e);

/* Solve to completion or until time_limit_s (<= 0: no limit) with initial
 * upper bound `ub` (INT32_MAX = +inf) and root row `root_perm` (NULL =
 * identity).  Leaves with cost < ub (<= with find_all) improve the bound. */
int pbb_solve(pbb_engine* e, int32_t ub, const int32_t* root_perm, double time_limit_s, pbb_result* out);

/* Resumable form: pbb_start bounds the root and unfolds the first path;
 * each pbb_explore runs the explorers for up to `seconds` of device time and
 * sets *done when the search space is exhausted. */
int pbb_start(pbb_engine* e, int32_t ub, const int32_t* root_perm);
int pbb_explore(pbb_engine* e, double seconds, int32_t* done);

/* Start on the factoradic interval [pos, end] (n digits each, digit i in
 * [0, n-i)): gpubb::initAtInterval (gpu/include/gpubb.h:155),
 * sequentialbb::initAtInterval (multicore/src/sequentialbb.cpp:84-106). */
int pbb_start_interval(pbb_engine* e, int32_t ub, const int32_t* root_perm, const int32_t* pos, const int32_t* end);

/* Start several explorers at once: interval k ([pos + k*n, end + k*n]) goes
 * to explorer ids[k] (ids NULL: explorer k); every explorer bounds the root
 * and unfolds its own start without counting, as initAtInterval does.
 * Replaces gpubb::initFromFac (gpu/include/gpubb.h:171, gpu/src/gpubb.cu:1245-1310)
 * and matrix_controller::initFromFac (multicore/include/matrix_controller.h:47).
 * nb_intervals in [1, nb_ivms]; ids distinct and < nb_ivms. */
int pbb_init_from_fac(pbb_engine* e, int32_t ub, const int32_t* root_perm, int32_t nb_intervals, const int32_t* ids,
                      const int32_t* pos, const int32_t* end);

/* Between windows (after pbb_explore returned): the intervals of the
 * explorers that still hold work, n digits each, with their explorer ids --
 * a checkpoint that pbb_init_from_fac resumes, in this engine or another.
 * Replaces gpubb::getIntervals (gpu/include/gpubb.h:172, gpu/src/gpubb.cu:1190-1242),
 * which also reports explorers by id.  PBB_E_INVAL when max_intervals is too
 * small (the reference exits there); counters are not reset. */
int pbb_get_intervals(pbb_engine* e, int32_t max_intervals, int32_t* pos, int32_t* end, int32_t* ids,
                      int32_t* nb_intervals);

/* Longest the host waits for one pbb_explore window (seconds): < 0 = the
 * window's device time + 60 s (default), 0 = no limit.  When the wait runs
 * out, pbb_explore returns PBB_E_TIMEOUT; the window still ends by its own
 * device-time budget, and the next call on the engine waits for it and
 * accounts for its work, so counters and intervals stay consistent. */
int pbb_set_wait_limit(pbb_engine* e, double seconds);

/* Checkpoint file of a search between windows, in the form the reference's
 * distributed master saves (works::save, distributed/src/works.cpp:172-190;
 * read back by works::init_infile :61-90): root solution, simple-bound
 * count, best solution, then one work whose intervals are the explorers'
 * (pbb_get_intervals) as decimal permutation indices (fact_work::VectToBigint,
 * distributed/src/fact_work.cpp:74-87).  pbb_load_checkpoint resumes such a
 * file in an engine of the same instance (pbb_init_from_fac with the best
 * makespan as the bound; the stored best schedule is reported when no leaf
 * improves it) and returns the stored bound count (may be NULL). */
int pbb_save_checkpoint(pbb_engine* e, const char* path);
int pbb_load_checkpoint(pbb_engine* e, const char* path, uint64_t* saved_simple_bounds);
/* A factoradic vector (n digits, digit i in [0, n-i)) as the decimal index
 * sum_i d_i (n-1-i)!, and back (indices below n!). */
int pbb_fact_to_decimal(int32_t n, const int32_t* digits, char* out, int32_t out_len);
int pbb_decimal_to_fact(int32_t n, const char* decimal, int32_t* digits);

/* Lower the incumbent to `ub` (a bound found by another solver; no
 * permutation is attached): solution::updateCost (common/src/solution.cpp:44-56). */
int pbb_set_ub(pbb_engine* e, int32_t ub);
int pbb_get_result(pbb_engine* e, pbb_result* out);

/* ------------------------------------------------------------------------
 * Pool: many instances resident on one GPU at once (batched solving and
 * continuous-batching serving).  No single counterpart in the reference; it
 * runs the same explorer as pbb_solve (gpubb::next, gpu/src/gpubb.cu:273-395)
 * for every resident instance inside one launch per window.
 *
 * Instances wait in a FIFO until a slot and enough explorer memory are free
 * (footprint per instance = explorers x (row stride^2 + 5 x row stride + 20
 * + 384 x row stride) bytes, row stride 32 for n <= 32 jobs, else 64).  Each pbb_pool_step
 * admits what fits, runs one exploration window of `window_s` device seconds
 * over all resident instances (one captured CUDA graph: explorer kernel,
 * status read-back), and retires the finished ones, whose results
 * pbb_pool_poll returns.  pbb_batch_solve admits the largest instances first.
 * ------------------------------------------------------------------------ */
typedef struct pbb_pool_config {
    int32_t device;
    int32_t max_jobs;            /* largest n accepted (<= 64); all instances share the row stride */
    int32_t max_machines;        /* largest m accepted (<= 32) */
    int32_t max_resident;        /* resident instances at most (0 = as many as CTAs fit) */
    int32_t warps_per_cta;       /* block shape: warps per CTA (0 = 8) */
    int32_t ctas_per_instance;   /* cap on the CTAs one instance gets in a window (0 = none); every
                                    window spreads all resident CTAs evenly over the instances */
    int32_t explorers_per_instance; /* explorers (IVMs) of each instance (0 = one per warp of the widest
                                       grid) */
    int32_t tail_warps;          /* block shape of the tail: once nothing waits and few instances remain,
                                    windows run CTAs of this many warps and last at least 20 ms (0 = 20;
                                    < 0 or <= warps_per_cta: no tail shape) */
    double window_s;             /* device time of one window (0 = 0.005) */
    int64_t explorer_bytes;      /* explorer memory budget (0 = 8 GiB) */
    int32_t core_warps;          /* work sharing of every instance, as pbb_config (0 = 8) */
    int32_t split_depth;         /* as pbb_config (0 = 10) */
    int32_t share_after;         /* as pbb_config (0 = 64; < 0 = at every step) */
    int32_t pad;
} pbb_pool_config;

typedef struct pbb_pool_result {
    int64_t tag;                 /* caller's tag of the submitted instance */
    int32_t windows;             /* windows the instance was resident */
    int32_t status;              /* PBB_OK, or an error code for this instance */
    pbb_result result;
} pbb_pool_result;

typedef struct pbb_pool pbb_pool;

void pbb_pool_config_default(pbb_pool_config* cfg);
int pbb_pool_create(const pbb_pool_config* cfg, pbb_pool** out);
int pbb_pool_destroy(pbb_pool* pool);
/* Queue an instance (copied) with its search settings (bounding/branching
 * mode, findAll, JohnsonMode of `search`; NULL = defaults), initial bound and
 * root permutation (NULL = identity). */
int pbb_pool_submit(pbb_pool* pool, const pbb_instance* inst, const pbb_config* search, int32_t ub,
                    const int32_t* root_perm, int64_t tag);
/* One window: admit, explore, retire.  Returns the counts left. */
int pbb_pool_step(pbb_pool* pool, int32_t* resident, int32_t* queued);
/* Move up to `max` finished results to `out`; *count = how many. */
int pbb_pool_poll(pbb_pool* pool, pbb_pool_result* out, int32_t max, int32_t* count);
/* Solve `count` instances to completion through one pool; results[i] for inst[i]. */
int pbb_batch_solve(const pbb_instance* inst, int32_t count, const pbb_config* search, const int32_t* ubs,
                    const pbb_pool_config* pool_cfg, pbb_result* results);

/* Children bounds of `count` nodes of one instance.  Node i is the schedule
 * sched[i*n .. i*n+n) with jobs [0..limit1[i]] fixed in front and
 * [limit2[i]..n) fixed at the back.  Per job id (0 for fixed jobs):
 * weak LB of the child with the job appended at the front / back
 * (bound_fsp_weak::boundChildren) and Johnson LB of the same children
 * (bound_fsp_strong::bornes_calculer on the child, no early exit).  Per node:
 * its own weak and Johnson LB (bornes_calculer); with at most one free job the
 * Johnson value is the makespan of the schedule as given.  Output arrays may
 * be NULL when not wanted. */
int pbb_bound_children(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t count,
                       const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                       int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                       int32_t* node_weak, int32_t* node_strong);

/* Outputs of pbb_bound_children_ex (host arrays; NULL = not wanted):
 * everything pbb_bound_children returns, plus the children's idle-time
 * priorities of the weak bound (prioBegin / prioEnd of
 * bound_fsp_weak::boundChildren, bounds/src/bound_fsp_weak.cpp:134-221) and
 * per node the idle time bound_fsp_strong::bornes_calculer returns in
 * couts[1] (bounds/src/bound_fsp_strong.cpp:457-509, 541-560: 0 when nothing
 * is fixed at the back, and 0 where the reference leaves it unset -- at most
 * one free job). */
typedef struct pbb_bound_out {
    int32_t *weak_begin, *weak_end, *strong_begin, *strong_end;   /* count x n, by job id */
    int32_t *node_weak, *node_strong;                             /* count */
    int32_t *prio_begin, *prio_end;                               /* count x n, by job id */
    int32_t *strong_idle;                                         /* count */
} pbb_bound_out;

int pbb_bound_children_ex(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t count,
                          const int32_t* sched, const int32_t* limit1, const int32_t* limit2, const pbb_bound_out* out);

/* pbb_bound_children for callers that cannot allocate GPU memory (a plugin
 * handed only device buffers, code running inside another framework's memory
 * pool).  No counterpart in the reference.  All node arrays are DEVICE
 * pointers owned by the caller; `stream` is a cudaStream_t (NULL = default
 * stream).  The only scratch (the instance tables and a status word) is a
 * 112 KiB static device array that every GPU loading the library keeps until
 * exit, so instances are limited to 64 jobs and 20 machines (larger ones:
 * PBB_E_INVAL).  The first call on a device looks the array up with
 * cudaGetSymbolAddress -- make it before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race, so do not issue them
 * concurrently (the function serialises its own host callers and waits for
 * `stream` before returning).  The calling thread's current device is left as
 * it was.  Outputs as pbb_bound_children; all required. */
int pbb_bound_children_noalloc(const pbb_instance* inst, int32_t johnson_mode, int32_t device, void* stream,
                               int32_t count, const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                               int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                               int32_t* node_weak, int32_t* node_strong);

/* NEH upper bound: jobs by decreasing total time, each inserted at the first
 * position of least partial makespan (host code). */
int pbb_neh(const pbb_instance* inst, int32_t* perm, int32_t* cost);

/* The same NEH on the device for `count` instances at once (one warp each,
 * Taillard's head/tail insertion: fastNEH::insertJobInBestPosition,
 * heuristic/src/fastNEH.cpp:206-220); results equal pbb_neh's.  perms has a
 * stride of PBB_MAX_JOBS per instance. */
int pbb_neh_batch(const pbb_instance* inst, int32_t count, int32_t device, int32_t* perms, int32_t* costs);

/* Iterated greedy from the NEH schedule on the device, one warp per instance
 * (IG::runIG, heuristic/src/IG.cpp:341-416): per round, 2 to 5 jobs removed
 * from a shuffled prefix of the middle-out visit order (:120-160), each put
 * back at its best position (:229-255), first-improvement insertion moves
 * within sqrt(n) places (localSearchKI :567-612), and the temperature
 * acceptance of 0.2 x mean time / 10 (:258-274) in the integer form
 * T / (T + delta).  Every random decision comes from the splitmix64 stream
 * seeded with seed + instance index, so a run is reproducible.  Same output
 * layout as pbb_neh_batch; the makespan never exceeds NEH's. */
int pbb_ig_batch(const pbb_instance* inst, int32_t count, int32_t device, int32_t iterations, uint64_t seed,
                 int32_t* perms, int32_t* costs);

#ifdef __cplusplus
}
#endif
#endif
