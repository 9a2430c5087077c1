// Host-callable launch wrappers of the engine kernels (pbb_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include "pbb_types.h"

namespace pbbl {
// dynamic shared memory of a CTA; fmask = 1 adds the explorer's per-warp
// free-position masks
int smem_bytes(int n, int m, int Ppad, int warps, int fmask = 0);
cudaError_t launch_reset(const DevGroup* groups, int ngroups, const int* ub, cudaStream_t st);
// reset must run first; interval b = g * per_group + j starts explorer j of
// group g, or explorer ids[b] when ids is given (distinct, < the explorer count)
cudaError_t launch_root(int nw, const DevGroup* groups, int ngroups, const int* roots, const int* ivals,
                        int root_stride, int smem, cudaStream_t st, int per_group = 1, const int* ids = nullptr);
cudaError_t launch_lower_ub(const DevGroup* groups, int g, int ub, cudaStream_t st);
// variant: 0 = no row sort, no early Johnson exit, no sampling (the hot
// path); 1 = each group's sortedDFS / earlyStopJohnson settings; 2 = as 1 and
// record sampled nodes (groups' SampleBuf); 3 = as 0 for groups that all
// bound in mode 2 with MinMin branching, without findAll, with position
// tables (all compiled in)
cudaError_t launch_explore(int nw, const DevGroup* groups, const int* ngroups_d, int ctas, int warps_per_cta, int smem,
                           unsigned long long budget_ns, int max_rounds, int select_budget, cudaStream_t st,
                           int variant = 0);
int explore_ctas_per_sm(int nw, int warps_per_cta, int smem, int variant = 0);
cudaError_t launch_bound(int nw, const DevInstance& I, int count, const int* sched, const int* l1, const int* l2,
                         int* wb, int* we, int* sb, int* se, int* nweak, int* nstrong, unsigned int* status, int ctas,
                         int warps_per_cta, int smem, cudaStream_t st, int method = 0, BoundExtra extra = BoundExtra());
}  // namespace pbbl
