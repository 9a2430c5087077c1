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
    int32_t n_jobs, n_machines, machine_pairs, explorers, warps, pad;
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

#ifdef __cplusplus
}
#endif
#endif
