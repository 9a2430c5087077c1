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
 * sweeps (nodes swept, free jobs summed over them, children they evaluated). */
typedef struct pbb_work {
    double device_seconds;
    int32_t n_jobs, n_machines, machine_pairs, explorers, warps, pad;
    uint64_t decomposed, simple_bounds, johnson_bounds;
    uint64_t johnson_sweeps, sweep_free_jobs, sweep_children;
} pbb_work;

struct pbb_engine;
int pbb_work_counters(struct pbb_engine* e, pbb_work* out);

#ifdef __cplusplus
}
#endif
#endif
