/*
 * pbbperm_diag.h -- diagnostics of libpbbperm.so (no counterpart in the
 * reference; used to state the engine's roofline).
 */
#ifndef PBBPERM_DIAG_H
#define PBBPERM_DIAG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Measured INT32 add+max throughput of `device` in Gop/s (all SMs, 2 ops
 * per step of independent register chains); `seconds` = kernel time. */
int pbb_diag_int32_peak(int32_t device, double* gops, double* seconds);

/* Work counters of an engine since its last start, for roofline accounting:
 * device time of the explorer kernels, bound evaluations, and the Johnson
 * sweeps (nodes swept, free jobs summed over them, children they evaluated)
 * and the direct per-child scans (children, free jobs summed over them). */
typedef struct pbb_work {
    double device_seconds;
    int32_t n_jobs, n_machines, machine_pairs, explorers, warps;
    int32_t status;                               /* PBB_ST_* bits the kernels raised */
    uint64_t decomposed, simple_bounds, johnson_bounds;
    uint64_t johnson_sweeps, sweep_free_jobs, sweep_children;
    uint64_t direct_children, direct_free_jobs;   /* children bounded by direct scans */
} pbb_work;

struct pbb_instance;

/* pbb_bound_children with the Johnson children evaluated by `method`:
 * 0 = forward/backward max-plus sweeps over all Johnson positions (what
 *     pbb_bound_children uses), 1 = direct per-child scans over the free
 *     positions (the explorer, for one or two children), 2 = the sweeps over
 *     the free positions only (the explorer, for more children).
 * Both must give the reference's values; tests compare them. */
int pbb_diag_bound_children(const struct pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t method,
                            int32_t count, const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                            int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                            int32_t* node_weak, int32_t* node_strong);

struct pbb_engine;
int pbb_work_counters(struct pbb_engine* e, pbb_work* out);

/* Status bit of pbb_work.status: 1 = a node the bound kernel rejected. */
#define PBB_DIAG_ST_BADINPUT 1

/* Limits of the explorer loop for tests of the bounded waits: at most
 * `select_budget` selection steps per explorer step (then the explorer
 * yields with its state consistent) and `max_rounds` loop rounds per window
 * launch (the window then ends early).  Defaults: 4096 and unbounded. */
int pbb_diag_set_step_limits(struct pbb_engine* e, int32_t select_budget, int32_t max_rounds);

/* Node sampling, for LB parity of the explorer's own bound code: from the
 * next pbb_explore on, the explorer records nodes it bounds -- those whose
 * hash of (explorer id, the warp's decomposed count) has its low `rate_log2`
 * bits clear -- until `capacity` records are taken (recording never waits).
 * capacity 0 turns sampling off.  A record is 8 + 5 n ints:
 *   [0] explorer id, [1] line (depth), [2] limit1, [3] limit2,
 *   [4] side chosen (0 front, 1 back), [5] incumbent when bounded,
 *   [6] free jobs, [7] 0,
 *   then n ints of schedule (front jobs, free jobs, back jobs: the
 *   reference's node->schedule), then n each of weak LB front, weak LB back,
 *   Johnson LB front, Johnson LB back, by job id, exactly as the explorer
 *   computed them before pruning (0 = not evaluated). */
int pbb_diag_sample_nodes(struct pbb_engine* e, int32_t capacity, int32_t rate_log2);
/* Copy up to max_records records; *count = records copied (max_records <= 0:
 * records available). */
int pbb_diag_get_samples(struct pbb_engine* e, int32_t max_records, int32_t* out, int32_t* count);

#ifdef __cplusplus
}
#endif
#endif
