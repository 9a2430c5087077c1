// Device heuristics (pbb_heur.cu): NEH and iterated greedy, one warp per
// instance.
#pragma once
#include <cuda_runtime.h>
#include "pbb_types.h"

// One instance for the heuristic kernels (device pointers).
struct NehTask {
    const int* p;   // [m][n] processing times
    int n, m;
    int* perm;      // [n] result permutation
    int* cost;      // result makespan (may be NULL)
    int* ub;        // also written here when not NULL (an explorer group's initial bound)
};

// Iterated greedy settings (pbb_ig_batch); the same stream of decisions on
// host and device for the same seed.
struct IgParams {
    int iterations;          // destruction / construction / local-search rounds
    int destruct;            // jobs removed per round at first (grows to destruct_max on failures)
    int destruct_max;
    int ls_passes;           // insertion local-search passes per round at most
    unsigned long long seed;
};

// shared memory of one heuristic block: p, heads, tails, and per-job arrays
#define PBB_HEUR_SMEM (int)(sizeof(int) * (PBB_MAX_N * PBB_MAX_M + PBB_MAX_N * 32 + (PBB_MAX_N + 1) * 32 + 6 * PBB_MAX_N))

namespace pbbl {
cudaError_t launch_neh(const NehTask* tasks_d, int count, cudaStream_t st);
cudaError_t launch_ig(const NehTask* tasks_d, int count, const IgParams& prm, cudaStream_t st);
}
