// Shared host/device definitions of the IVM flow-shop engine.
#pragma once
#include <stdint.h>

#define PBB_MAX_N 64          // jobs per instance (int8 IVM cells, two 32-bit mask words)
#define PBB_MAX_M 32          // machines per instance (one machine per lane in recurrences)
#define PBB_WARPS_MAX 20      // explorer warps per CTA (96 registers a thread)
#define PBB_CORE_WARPS 8      // default of DevSearch::core_warps
#define PBB_SPLIT_DEPTH 10    // default of DevSearch::split_depth
#define PBB_SHARE_AFTER 64    // default of DevSearch::share_after

// IVM life cycle (per explorer, in global memory)
#define IVM_IDLE 0            // no interval
#define IVM_QUEUED 1          // registered in the idle queue, waiting for a donor
#define IVM_ACTIVE 2          // holds a non-empty interval

// status bits written by kernels (never traps)
#define PBB_ST_BADINPUT 1u    // a node or instance the kernel rejected

// Packed Johnson entry for (pair i, Johnson position t):
//   bits 0..15 p[m0][job], 16..31 p[m1][job], 32..39 job id, 40..63 lag[i][job]
// (the two processing times share the low word, so the scans unpack them with
// one mask and one shift)
#define JE_PACK(job, a, b, lag) ((unsigned long long)(a) | ((unsigned long long)(b) << 16) | \
                                 ((unsigned long long)(job) << 32) | ((unsigned long long)(lag) << 40))
#define JE_A(e) ((int)((unsigned)(e) & 0xFFFFu))
#define JE_B(e) ((int)((unsigned)(e) >> 16))
#define JE_JOB(e) ((int)(((e) >> 32) & 0xFFull))
#define JE_C(e) ((int)((e) >> 40))

// One flow-shop instance as the kernels see it (device pointers).
struct DevInstance {
    int n, m;
    int P;        // machine pairs used by the Johnson bound
    int Ppad;     // P rounded up to 32
    const int* p;                    // [m][n]
    const unsigned long long* je;    // [n][Ppad]
    const unsigned char* posj;       // [n][Ppad] Johnson position of each job per pair (may be NULL)
    const unsigned char* pm0;        // [Ppad]
    const unsigned char* pm1;        // [Ppad]
    const int* min_arr;              // [m]
    const int* min_dep;              // [m]
};

// Search settings shared by a group of explorers.
struct DevSearch {
    int bound_mode;    // 0 weak, 1 strong, 2 weak then strong
    int branch_mode;   // -3,-2,-1 fixed; 1 MaxSum, 2 MinBranch, 3 MinMin
    int find_all;
    int sort_nodes;    // [bb] sortedDFS: 0 reverse the row on a side change, 1 sort it by cost,
                       //      2 and 4 by (cost, priority), 3 by priority
    int sort_crit;     // [bb] sortingCriterion (sortedDFS >= 2): 1 cost, 2 cost minus the other side's, 3 idle time
    int early_stop;    // [bb] earlyStopJohnson: a child's Johnson scan may stop once it exceeds the incumbent
    int core_warps;    // warps per CTA that ask for work whatever the search's width (1..warps per CTA)
    int split_depth;   // work is not split at levels deeper than n - split_depth
    int share_after;   // an explorer offers work only after decomposing this many nodes since it got
                       // its interval or last gave part of it away (0 = at every step)
};

// Per-group control block (device memory).
// The fields every warp polls or updates under contention each sit on their
// own 128-byte line, so that reads of the incumbent and of the active count
// do not queue behind the idle-queue atomics (and the other way round).
struct GroupCtl {
    alignas(128) unsigned long long best_key;   // (cost << 32) | ivm id of the slot holding the permutation
    alignas(128) int active;                    // explorers holding work
    alignas(128) unsigned long long q_head;     // idle-explorer queue cursors
    alignas(128) unsigned long long q_tail;
    alignas(128) int found;                     // leaves that improved (or matched, with findAll) the bound
    unsigned int status;                        // PBB_ST_* bits
    unsigned long long decomposed, johnson_bounds, simple_bounds, leaves, root_simple;
    unsigned long long steals;                  // intervals handed over
    // work of the Johnson sweeps: nodes swept, free jobs summed over them,
    // children evaluated by them (roofline accounting)
    unsigned long long jsweeps, jfree, jchild;
    // children bounded by direct scans, and their free jobs summed
    unsigned long long jdirect, jdirect_free;
};

// Explorer storage of a group (device memory, structure of arrays).
struct DevIvms {
    int count;             // explorers in the group
    int npad;              // row stride (64)
    signed char* mat;      // [count][npad][npad]
    signed char* pos;      // [count][npad]
    signed char* end;      // [count][npad]
    signed char* dir;      // [count][npad]
    signed char* pj;       // [count][npad] job fixed at each level of the current path
    int* line;             // [count]
    int* state;            // [count]
    int* bestcost;         // [count]
    signed char* bestperm; // [count][npad]
    unsigned int* qseq;    // [count] Vyukov queue cell sequence numbers
    int* qval;             // [count] queued explorer ids
    int* path;             // [count][npad levels][3][32] heads / tails / free loads of the path nodes
};

#define PBB_PATH_INTS 96   // ints per path level: heads, tails, free loads, 32 machines each

// Opt-in record of nodes the explorer bounded, as it bounded them (LB parity
// of the explorer's own bound code).  A node is recorded when a hash of
// (explorer id, the warp's decomposed count) has its low bits clear under
// rate_mask, until `cap` records are taken; recording never waits.
// Record layout (ints): PBB_SAMPLE_HDR header
//   [0] explorer id  [1] line  [2] limit1  [3] limit2  [4] side chosen
//   [5] incumbent at bounding  [6] free jobs k  [7] 0
// then five arrays of n: schedule (front jobs, free jobs, back jobs as the
// reference's node->schedule), weak LB front / back and Johnson LB front /
// back by job id (0 = not evaluated).
#define PBB_SAMPLE_HDR 8
struct SampleBuf {
    unsigned count;        // records claimed (may exceed cap; only cap are written)
    unsigned cap;
    unsigned rate_mask;
    int stride;            // ints per record: PBB_SAMPLE_HDR + 5 n
    int* rec;
};

struct DevGroup {
    DevInstance inst;
    DevSearch search;
    DevIvms ivm;
    GroupCtl* ctl;
    int first_cta;         // CTAs [first_cta, first_cta + ctas) work on this group
    int ctas;
    SampleBuf* sample;     // NULL unless node sampling is armed
};

// Optional outputs of the bound kernel (NULL = not wanted): per node and job,
// the children's idle-time priorities, and per node the Johnson bound's idle
// time of the fixed jobs.
struct BoundExtra {
    int* prio_begin = nullptr;   // [count][n]
    int* prio_end = nullptr;     // [count][n]
    int* strong_idle = nullptr;  // [count]
};

// Dynamic shared memory layout of one CTA (host and device agree).
struct SmemPlan {
    int je_off, p_off, pm0_off, pm1_off, marr_off, mdep_off, posj_off, warp_off, warp_bytes, total;
    int fmask;             // 1: each warp keeps its explorer's free-position masks (explorer only)
};

__host__ __device__ inline int pbb_align(int x, int a) { return (x + a - 1) / a * a; }

// per-warp scratch: [fmask: u64 fmask[Ppad]] ints lbF[n] lbB[n] frontZ backZ
// Fb Bb rem RB FR [32 each]; shorts dF[n*m] dB[n*m]; bytes fjob[n] bjob[n] row[n]
__host__ __device__ inline int pbb_warp_bytes(int n, int m, int Ppad, int fmask)
{
    return pbb_align((fmask ? Ppad * 8 : 0) + (2 * n + 7 * 32) * 4 + 2 * n * m * 2 + 3 * n, 16);
}

__host__ __device__ inline SmemPlan pbb_smem_plan(int n, int m, int Ppad, int warps, int fmask = 0)
{
    SmemPlan s;
    int off = 0;
    s.je_off = off;   off += n * Ppad * 8;
    s.p_off = off;    off += pbb_align(m * n * 4, 16);
    s.pm0_off = off;  off += pbb_align(Ppad, 16);
    s.pm1_off = off;  off += pbb_align(Ppad, 16);
    s.marr_off = off; off += pbb_align(m * 4, 16);
    s.mdep_off = off; off += pbb_align(m * 4, 16);
    s.posj_off = off; off += pbb_align(n * Ppad, 16);
    s.warp_off = off;
    s.fmask = fmask;
    s.warp_bytes = pbb_warp_bytes(n, m, Ppad, fmask);
    off += s.warp_bytes * warps;
    s.total = off;
    return s;
}
