// Kernels of the IVM flow-shop engine (sm_100a).
//
//   pbb_reset_kernel     explorers empty, idle queue and counters cleared
//   pbb_root_kernel      root row bounded (weak, uncounted) + initial unfold
//   pbb_explore_kernel   persistent explorer loop: select/decode/bound/prune
//                        and work sharing through a device idle queue
//   pbb_bound_kernel     batched children bounds of given nodes (LB parity API)
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include "pbb_types.h"
#include "pbb_device.cuh"
#include "pbb_launch.h"

using namespace pbb;

namespace {

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p)
{
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}

__device__ __forceinline__ int ld_volatile_s32(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

// Load the group's instance tables into this CTA's shared memory.
__device__ __forceinline__ void load_tables(const DevInstance& I, unsigned char* smem, const SmemPlan& sp, CtaTables& T)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    unsigned long long* je = reinterpret_cast<unsigned long long*>(smem + sp.je_off);
    int* p = reinterpret_cast<int*>(smem + sp.p_off);
    unsigned char* pm0 = smem + sp.pm0_off;
    unsigned char* pm1 = smem + sp.pm1_off;
    int* marr = reinterpret_cast<int*>(smem + sp.marr_off);
    int* mdep = reinterpret_cast<int*>(smem + sp.mdep_off);
    for (int i = tid; i < I.n * I.Ppad; i += nt) je[i] = I.je[i];
    for (int i = tid; i < I.n * I.m; i += nt) p[i] = I.p[i];
    for (int i = tid; i < I.Ppad; i += nt) { pm0[i] = I.pm0[i]; pm1[i] = I.pm1[i]; }
    for (int i = tid; i < I.m; i += nt) { marr[i] = I.min_arr[i]; mdep[i] = I.min_dep[i]; }
    unsigned char* posj = smem + sp.posj_off;
    if (I.posj)
        for (int i = tid; i < I.n * I.Ppad; i += nt) posj[i] = I.posj[i];
    T.je = je; T.p = p; T.pm0 = pm0; T.pm1 = pm1; T.min_arr = marr; T.min_dep = mdep;
    T.posj = I.posj ? posj : nullptr;
    T.n = I.n; T.m = I.m; T.P = I.P; T.Ppad = I.Ppad;
}

// ---------------------------------------------------------------------------
// explorer registers and their HBM image
// ---------------------------------------------------------------------------
template <int NW>
struct Ivm {
    int pos[NW], end[NW], dir[NW], pj[NW], row[NW];
    int line;
    int hf, hb, hr;   // partial schedule of the node at `line`, lane = machine
};

__device__ __forceinline__ int* path_level(const DevIvms& V, int id, int l)
{
    return V.path + ((size_t)id * V.npad + l) * PBB_PATH_INTS;
}

template <int NW>
__device__ __forceinline__ void load_path(const DevIvms& V, int id, int l, Ivm<NW>& R)
{
    const int* q = path_level(V, id, l) + lane_id();
    R.hf = __ldcg(q);
    R.hb = __ldcg(q + 32);
    R.hr = __ldcg(q + 64);
}

template <int NW>
__device__ __forceinline__ void store_path(const DevIvms& V, int id, int l, const Ivm<NW>& R)
{
    int* q = path_level(V, id, l) + lane_id();
    __stcg(q, R.hf);
    __stcg(q + 32, R.hb);
    __stcg(q + 64, R.hr);
}

// path vectors of level L+1 from those of level L, job u fixed on side dir
template <int NW>
__device__ __forceinline__ void path_down(const CtaTables& T, Ivm<NW>& R, int u, int dir)
{
    if (dir == 0) R.hf = append_front(T, R.hf, u);
    else R.hb = prepend_back(T, R.hb, u);
    if (lane_id() < T.m) R.hr -= T.p[lane_id() * T.n + u];
}

// jobs fixed in front among the levels above L
template <int NW>
__device__ __forceinline__ int front_count(const Ivm<NW>& R, int L)
{
    int f = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int lv = w * 32 + lane_id();
        f += __popc(__ballot_sync(FULLMASK, lv < L && R.dir[w] == 0));
    }
    return f;
}

__device__ __forceinline__ signed char* mat_row(const DevIvms& V, int id, int l)
{
    return V.mat + ((size_t)id * V.npad + l) * V.npad;
}

template <int NW>
__device__ __forceinline__ void load_row(const DevIvms& V, int id, int l, int (&row)[NW])
{
    const signed char* r = mat_row(V, id, l);
#pragma unroll
    for (int w = 0; w < NW; w++) row[w] = __ldcg(r + w * 32 + lane_id());
}

template <int NW>
__device__ __forceinline__ void store_row(const DevIvms& V, int id, int l, const int (&row)[NW])
{
    signed char* r = mat_row(V, id, l);
#pragma unroll
    for (int w = 0; w < NW; w++) __stcg(r + w * 32 + lane_id(), (signed char)row[w]);
}

template <int NW>
__device__ __forceinline__ void load_ivm(const DevIvms& V, int id, Ivm<NW>& R)
{
    const size_t b = (size_t)id * V.npad;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int e = w * 32 + lane_id();
        R.pos[w] = __ldcg(V.pos + b + e);
        R.end[w] = __ldcg(V.end + b + e);
        R.dir[w] = __ldcg(V.dir + b + e);
        R.pj[w] = __ldcg(V.pj + b + e);
    }
    R.line = __ldcg(V.line + id);
    load_row<NW>(V, id, R.line, R.row);
    load_path<NW>(V, id, R.line, R);
}

template <int NW>
__device__ __forceinline__ void store_ivm(const DevIvms& V, int id, const Ivm<NW>& R)
{
    const size_t b = (size_t)id * V.npad;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int e = w * 32 + lane_id();
        __stcg(V.pos + b + e, (signed char)R.pos[w]);
        __stcg(V.end + b + e, (signed char)R.end[w]);
        __stcg(V.dir + b + e, (signed char)R.dir[w]);
        __stcg(V.pj + b + e, (signed char)R.pj[w]);
    }
    if (lane_id() == 0) __stcg(V.line + id, R.line);
}

// front / back job lists of the current path (ivm_bound.cpp:112-138)
template <int NW>
__device__ __forceinline__ void build_lists(const WarpScratch& S, const Ivm<NW>& R, int L, int& f, int& b)
{
    f = 0; b = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int lv = w * 32 + lane_id();
        const bool isF = lv < L && R.dir[w] == 0;
        const bool isB = lv < L && R.dir[w] != 0;
        const unsigned bf = __ballot_sync(FULLMASK, isF), bb = __ballot_sync(FULLMASK, isB);
        if (isF) S.fjob[f + __popc(bf & lanemask_lt())] = (unsigned char)R.pj[w];
        if (isB) S.bjob[b + __popc(bb & lanemask_lt())] = (unsigned char)R.pj[w];
        f += __popc(bf);
        b += __popc(bb);
    }
    __syncwarp();
}

// 32-bit per warp (fewer live registers in the explorer loop), added to the
// group's 64-bit counters at least every 2^20 decomposed nodes
struct WarpCounters {
    unsigned decomposed, simple, johnson, leaves;
    unsigned sweeps, free_jobs, swept_children, direct_children, direct_free;
};

__device__ __forceinline__ void flush_counters(const DevGroup& G, WarpCounters& C)
{
    if (lane_id() == 0) {
        atomicAdd(&G.ctl->decomposed, (unsigned long long)C.decomposed);
        atomicAdd(&G.ctl->simple_bounds, (unsigned long long)C.simple);
        atomicAdd(&G.ctl->johnson_bounds, (unsigned long long)C.johnson);
        atomicAdd(&G.ctl->leaves, (unsigned long long)C.leaves);
        atomicAdd(&G.ctl->jsweeps, (unsigned long long)C.sweeps);
        atomicAdd(&G.ctl->jfree, (unsigned long long)C.free_jobs);
        atomicAdd(&G.ctl->jchild, (unsigned long long)C.swept_children);
        atomicAdd(&G.ctl->jdirect, (unsigned long long)C.direct_children);
        atomicAdd(&G.ctl->jdirect_free, (unsigned long long)C.direct_free);
    }
    C = WarpCounters{0, 0, 0, 0, 0, 0, 0, 0, 0};
}

// Record an improving leaf: permutation into the explorer's slot, then the
// (cost, explorer) key into the group's best (solution.cpp:27-45 restated as
// a packed atomicMin instead of a mutex).
template <int NW>
__device__ __forceinline__ void record_solution(const DevGroup& G, const WarpScratch& S, int id, int f, int b, int last, int cost)
{
    const int n = G.inst.n;
    signed char* slot = G.ivm.bestperm + (size_t)id * G.ivm.npad;
    for (int i = lane_id(); i < n; i += 32) {
        int j;
        if (i < f) j = S.fjob[i];
        else if (i == f) j = last;
        else j = S.bjob[n - 1 - i];
        slot[i] = (signed char)j;
    }
    __syncwarp();
    if (lane_id() == 0) {
        G.ivm.bestcost[id] = cost;
        __threadfence();
        atomicMin(&G.ctl->best_key, ((unsigned long long)(unsigned)cost << 32) | (unsigned)id);
        atomicAdd(&G.ctl->found, 1);
    }
    __syncwarp();
}

// One call of sequentialbb::next (multicore/src/sequentialbb.cpp:110-190):
// advance to the next unpruned node of the interval, evaluating leaves on the
// way.  Returns 1 with a node to bound at R.line, 0 when the interval is
// exhausted, 2 when the selection budget ran out (state stays consistent).
template <int NW, int FM = 0>
__device__ __forceinline__ int select_node(const DevGroup& G, const CtaTables& T, const WarpScratch& S, int id, Ivm<NW>& R,
                           int& best, WarpCounters& C, int budget)
{
    const int n = T.n;
    const bool fa = G.search.find_all != 0;
    for (int it = 0; it < budget; it++) {
        if (!before_end<NW>(R.pos, R.end, n)) return 0;
        int L = R.line;
        const int k = n - L;
        const int p = vget<NW>(R.pos, L);
        if (p >= k) {                                    // goUp (ivm.cpp:56-72)
            if (L > 0) {
                vset<NW>(R.pos, L, 0);
                L--;
                R.line = L;
                if (FM || S.fmask) fmask_flip(T, S, vget<NW>(R.pj, L));   // its job is free again
                load_row<NW>(G.ivm, id, L, R.row);
                load_path<NW>(G.ivm, id, L, R);
                const int pp = vget<NW>(R.pos, L);
                if (lane_id() == (pp & 31)) {
#pragma unroll
                    for (int w = 0; w < NW; w++)
                        if ((pp >> 5) == w) {
                            R.row[w] = cell_flag(R.row[w]);
                            __stcg(mat_row(G.ivm, id, L) + pp, (signed char)R.row[w]);
                        }
                }
            } else {
                vset<NW>(R.pos, 0, p + 1);
            }
            continue;
        }
        int q = next_open_cell<NW>(R.row, p, k);         // goRight over pruned cells
        if (q != p) {
            vset<NW>(R.pos, L, q);
            // an open cell was found: go down into it in this same step, as
            // the next iteration would (the interval end is checked again)
            if (q >= k) continue;
            if (!before_end<NW>(R.pos, R.end, n)) return 0;
        }
        // goDown (ivm.cpp:73-104): the node at (L, q) is decomposed
        C.decomposed++;
        const int u = vget<NW>(R.row, q);
        vset<NW>(R.pj, L, u);
        if (FM || S.fmask) fmask_flip(T, S, u);                  // u is fixed below this level
        path_down<NW>(T, R, u, vget<NW>(R.dir, L));
        int nr[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int idx = w * 32 + lane_id();
            int src = idx < q ? idx : idx + 1;
            if (src >= 32 * NW) src = 0;
            nr[w] = cell_job(vgather<NW>(R.row, src));
        }
#pragma unroll
        for (int w = 0; w < NW; w++) R.row[w] = nr[w];
        L++;
        R.line = L;
        vset<NW>(R.pos, L, 0);
        vset<NW>(R.dir, L, 0);
        store_path<NW>(G.ivm, id, L, R);
        if (L == n - 1) {                                 // leaf (ivm_bound.cpp:239-271)
            C.leaves++;
            const int f0 = front_count<NW>(R, L);
            const int last = vget<NW>(R.row, 0);
            partial_from_path(T, S, f0, L - f0, R.hf, R.hb, R.hr);
            int cost = 0;
            if (lane_id() == 0) cost = makespan_split(T, S, last, -1);
            cost = __shfl_sync(FULLMASK, cost, 0);
            const bool better = fa ? !(cost > best) : !(cost >= best);
            if (better) {
                best = cost;
                int f, b;
                build_lists<NW>(S, R, L, f, b);
                record_solution<NW>(G, S, id, f, b, last, cost);
            }
            if (lane_id() == 0) {
                R.row[0] = cell_flag(R.row[0]);
                __stcg(mat_row(G.ivm, id, L), (signed char)R.row[0]);
            }
            continue;
        }
        return 1;
    }
    return 2;
}

// Node sampling (SampleBuf): claim a record for the node about to be bounded
// when the hash of (explorer, the warp's decomposed count) falls under the
// group's rate, and write its header and fixed jobs; NULL when not sampled or
// when the buffer is full (recording never waits).
template <int NW>
__device__ __forceinline__ int* sample_slot(const DevGroup& G, const WarpScratch& S, const Ivm<NW>& R, int id, int f,
                                            int b, int best, unsigned long long step)
{
    SampleBuf* sb = G.sample;
    int slot = -1;
    if (lane_id() == 0 && sb) {
        unsigned h = (unsigned)id * 0x9E3779B1u ^ (unsigned)step * 0x85EBCA77u;
        h ^= h >> 15;
        h *= 0x2C1B3C6Du;
        h ^= h >> 12;
        h *= 0x297A2D39u;
        h ^= h >> 15;
        if ((h & sb->rate_mask) == 0) {
            const unsigned c = atomicAdd(&sb->count, 1u);
            if (c < sb->cap) slot = (int)c;
        }
    }
    slot = __shfl_sync(FULLMASK, slot, 0);
    if (slot < 0) return nullptr;
    int* rec = sb->rec + (size_t)slot * sb->stride;
    const int n = G.inst.n, L = R.line;
    int fc = 0, bc = 0;
    build_lists<NW>(S, R, L, fc, bc);
    int* sch = rec + PBB_SAMPLE_HDR;
    for (int i = lane_id(); i < f; i += 32) sch[i] = S.fjob[i];
    for (int i = lane_id(); i < b; i += 32) sch[n - 1 - i] = S.bjob[i];
    if (lane_id() == 0) {
        rec[0] = id;
        rec[1] = L;
        rec[2] = f - 1;
        rec[3] = n - b;
        rec[5] = best;
        rec[6] = n - L;
        rec[7] = 0;
    }
    __syncwarp();
    return rec;
}

// Bound and prune the node selected at R.line and write its row back.
template <int NW, int SORT, int SAMPLE, int RULE>
__device__ __forceinline__ void bound_current(const DevGroup& G, const CtaTables& T, const WarpScratch& S, int id,
                                              Ivm<NW>& R, int mode, int best, WarpCounters& C)
{
    const int L = R.line;
    const int f = front_count<NW>(R, L), b = L - f;
    partial_from_path(T, S, f, b, R.hf, R.hb, R.hr);
    const int prev = L > 0 ? vget<NW>(R.dir, L - 1) : 0;
    int* rec = nullptr;
    if (SAMPLE) rec = sample_slot<NW>(G, S, R, id, f, b, best, C.decomposed);
    NodeCounters nc = {0, 0, 0, 0, 0};
    const int d = bound_and_prune<NW, SORT, SAMPLE, RULE>(T, S, G.search, mode, R.row, T.n - L, f, b, L, prev, best, nc,
                                                    true, rec);
    vset<NW>(R.dir, L, d);
    store_row<NW>(G.ivm, id, L, R.row);
    C.simple += (unsigned)nc.simple;
    C.johnson += (unsigned)nc.johnson;
    C.sweeps += (unsigned)nc.sweeps;
    C.free_jobs += (unsigned)nc.free_jobs;
    C.swept_children += (unsigned)nc.swept_children;
    C.direct_children += (unsigned)nc.direct_children;
    C.direct_free += (unsigned)nc.direct_free;
}

// ---------------------------------------------------------------------------
// idle-explorer queue: bounded MPMC queue with per-cell sequence numbers
// (D. Vyukov's design), one lane operates it
// ---------------------------------------------------------------------------
__device__ bool queue_push(const DevGroup& G, int v)
{
    const unsigned long long cap = (unsigned long long)G.ivm.count;
    for (int attempt = 0; attempt < 64; attempt++) {
        unsigned long long pos = ld_volatile_u64(&G.ctl->q_tail);
        const int cell = (int)(pos % cap);
        const unsigned seq = ld_acquire_u32(G.ivm.qseq + cell);
        const int dif = (int)(seq - (unsigned)pos);
        if (dif == 0) {
            if (atomicCAS(&G.ctl->q_tail, pos, pos + 1) == pos) {
                G.ivm.qval[cell] = v;
                st_release_u32(G.ivm.qseq + cell, (unsigned)(pos + 1));
                return true;
            }
        } else if (dif < 0) {
            return false;
        }
    }
    return false;
}

__device__ int queue_pop(const DevGroup& G)
{
    const unsigned long long cap = (unsigned long long)G.ivm.count;
    for (int attempt = 0; attempt < 64; attempt++) {
        unsigned long long pos = ld_volatile_u64(&G.ctl->q_head);
        const int cell = (int)(pos % cap);
        const unsigned seq = ld_acquire_u32(G.ivm.qseq + cell);
        const int dif = (int)(seq - (unsigned)(pos + 1));
        if (dif == 0) {
            if (atomicCAS(&G.ctl->q_head, pos, pos + 1) == pos) {
                const int v = __ldcg(G.ivm.qval + cell);
                st_release_u32(G.ivm.qseq + cell, (unsigned)(pos + cap));
                return v;
            }
        } else if (dif < 0) {
            return -1;
        }
    }
    return -1;
}

// Split the explorer's interval with a queued idle explorer
// (bbthread::shareWork multicore/src/bbthread.cpp:40-72 and
// ivm::cuttingPosition multicore/src/ivm.cpp:199-237): the first level l where
// pos and end differ (not below the current line, not deeper than n-10) is
// cut so that the donor keeps half of the explorable cells after pos[l]; the
// receiver gets row l, the path vectors of level l and the right part, and
// continues with next() without an uncounted unfold, so decomposed-node counts
// do not depend on how the work was shared.
template <int NW>
__device__ __forceinline__ int try_share(const DevGroup& G, int id, Ivm<NW>& R)
{
    const int n = G.inst.n;
    // cheap emptiness test of the queue first (one lane reads, all follow)
    int empty = 0;
    if (lane_id() == 0) empty = ld_volatile_u64(&G.ctl->q_tail) == ld_volatile_u64(&G.ctl->q_head);
    if (__shfl_sync(FULLMASK, empty, 0)) return 0;
    int f = n;
#pragma unroll
    for (int w = NW - 1; w >= 0; w--) {
        const int lv = w * 32 + lane_id();
        const unsigned d = __ballot_sync(FULLMASK, lv < n && R.pos[w] != R.end[w]);
        if (d) f = w * 32 + __ffs(d) - 1;
    }
    const int lcap = max(n - G.search.split_depth, 0);
    int l = f;
    if (l > R.line) l = R.line;
    if (l > lcap) l = lcap;
    const int pl = vget<NW>(R.pos, l), el = vget<NW>(R.end, l);
    if (!(pl < el)) return 0;

    int row[NW];
    if (l == R.line) {
#pragma unroll
        for (int w = 0; w < NW; w++) row[w] = R.row[w];
    } else {
        load_row<NW>(G.ivm, id, l, row);
    }
    // cutting position: keep = explorable / 2 cells after pos[l]
    int expl = 0;
    unsigned em[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int idx = w * 32 + lane_id();
        em[w] = __ballot_sync(FULLMASK, idx > pl && idx <= el && row[w] >= 0);
        expl += __popc(em[w]);
    }
    // nothing explorable after pos[l]: a receiver would only skip pruned
    // cells.  Instead the donor drops those cells from its own interval
    // (end[l] = pos[l], levels below l open to their last cell), which removes
    // no node that could be decomposed and lets the next split look deeper.
    if (expl == 0) {
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int lv = w * 32 + lane_id();
            if (lv == l) R.end[w] = pl;
            else if (lv > l) R.end[w] = n - 1 - lv;
        }
        return 2;
    }
    int thief = -1;
    if (lane_id() == 0) thief = queue_pop(G);
    thief = __shfl_sync(FULLMASK, thief, 0);
    if (thief < 0) return 0;
    const int keep = expl / 2;
    int cut = pl + 1;
    if (keep > 0) {
        int rem = keep;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int c = __popc(em[w]);
            if (rem > 0 && rem <= c) {
                unsigned msk = em[w];
                for (int r = 1; r < rem; r++) msk &= msk - 1;
                cut = w * 32 + __ffs(msk) - 1 + 1;
                rem = 0;
            } else if (rem > 0) {
                rem -= c;
            }
        }
    }
    // receiver image.  Above level l the receiver's pos equals its end, so it
    // never decomposes a node there: going up to l-1 it only flags the cell
    // it came from and finds its interval exhausted.  Row l and the path
    // vectors of level l are therefore all it reads of the donor's stack.
    const size_t tb = (size_t)thief * G.ivm.npad;
    store_row<NW>(G.ivm, thief, l, row);
    {
        const int* ps = path_level(G.ivm, id, l) + lane_id();
        int* pd = path_level(G.ivm, thief, l) + lane_id();
        const int a = __ldcg(ps), b = __ldcg(ps + 32), c = __ldcg(ps + 64);
        __stcg(pd, a);
        __stcg(pd + 32, b);
        __stcg(pd + 64, c);
    }
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int lv = w * 32 + lane_id();
        const int tp = lv < l ? R.pos[w] : (lv == l ? cut : 0);
        __stcg(G.ivm.pos + tb + lv, (signed char)tp);
        __stcg(G.ivm.end + tb + lv, (signed char)R.end[w]);
        __stcg(G.ivm.dir + tb + lv, (signed char)(lv <= l ? R.dir[w] : 0));
        __stcg(G.ivm.pj + tb + lv, (signed char)(lv < l ? R.pj[w] : 0));
    }
    if (lane_id() == 0) __stcg(G.ivm.line + thief, l);
    // donor keeps [pos, cut-1] at level l, everything below l
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int lv = w * 32 + lane_id();
        if (lv == l) R.end[w] = cut - 1;
        else if (lv > l) R.end[w] = n - 1 - lv;
    }
    __threadfence();
    __syncwarp();
    if (lane_id() == 0) {
        atomicAdd(&G.ctl->active, 1);
        atomicAdd(&G.ctl->steals, 1ull);
        st_release(G.ivm.state + thief, IVM_ACTIVE);
    }
    __syncwarp();
    return 1;
}

__device__ __forceinline__ int group_of_cta(const DevGroup* groups, int ngroups)
{
    int lo = 0, hi = ngroups - 1;
    const int c = blockIdx.x;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (groups[mid].first_cta <= c) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// Empty every explorer of every group; clear counters and queues.
__global__ void pbb_reset_kernel(const DevGroup* groups, int ngroups, const int* ub)
{
    for (int g = blockIdx.y; g < ngroups; g += gridDim.y) {
        const DevGroup G = groups[g];
        const int n = G.inst.n;
        for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < G.ivm.count; id += gridDim.x * blockDim.x) {
            G.ivm.state[id] = IVM_IDLE;
            G.ivm.line[id] = 0;
            G.ivm.bestcost[id] = 0x7fffffff;
            G.ivm.qseq[id] = (unsigned)id;
            const size_t b = (size_t)id * G.ivm.npad;
            for (int e = 0; e < G.ivm.npad; e++) {
                G.ivm.pos[b + e] = 0;
                G.ivm.end[b + e] = 0;
                G.ivm.dir[b + e] = 0;
                G.ivm.pj[b + e] = 0;
            }
            G.ivm.pos[b] = (signed char)n;   // empty interval (ivm.cpp:36-49)
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            GroupCtl* c = G.ctl;
            c->best_key = ((unsigned long long)(unsigned)ub[g] << 32) | 0xffffffffull;
            c->active = 0; c->found = 0; c->status = 0;
            c->decomposed = c->johnson_bounds = c->simple_bounds = c->leaves = c->root_simple = 0;
            c->q_head = c->q_tail = 0; c->steals = 0;
            c->jsweeps = c->jfree = c->jchild = 0;
            c->jdirect = c->jdirect_free = 0;
        }
    }
}

// Root of each group (one warp per group): row 0 = root permutation, bounded
// with the weak bound and pruned without counting (ivm_bound::boundRoot
// ivm_bound.cpp:274-336, stats reset by initAtInterval sequentialbb.cpp:84-106),
// then the uncounted descent along the interval start (unfold :207-264).
template <int NW>
__global__ void pbb_root_kernel(const DevGroup* groups, int ngroups, const int* roots, const int* ivals,
                                int root_stride, int per_group, const int* ids)
{
    extern __shared__ __align__(16) unsigned char smem[];
    // block b starts explorer ids[b] (b % per_group without ids) of group
    // b / per_group on interval b
    const int b = blockIdx.x;
    const int g = b / per_group;
    if (g >= ngroups) return;
    const DevGroup G = groups[g];
    const SmemPlan sp = pbb_smem_plan(G.inst.n, G.inst.m, G.inst.Ppad, 1);
    CtaTables T;
    load_tables(G.inst, smem, sp, T);
    __syncthreads();
    const WarpScratch S = warp_scratch(smem + sp.warp_off, sp, T.n, T.m, T.Ppad);
    const int n = T.n;
    const int id = ids ? ids[b] : b % per_group;
    Ivm<NW> R;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int e = w * 32 + lane_id();
        // interval [pos, end] of this explorer (initAtInterval sequentialbb.cpp:84-106)
        R.pos[w] = e < n ? ivals[(2 * b) * root_stride + e] : 0;
        R.end[w] = e < n ? ivals[(2 * b + 1) * root_stride + e] : 0;
        R.dir[w] = 0;
        R.pj[w] = 0;
        R.row[w] = e < n ? roots[g * root_stride + e] : 0;
    }
    R.line = 0;
    int best = (int)(G.ctl->best_key >> 32);
    NodeCounters rootc = {0, 0, 0, 0, 0};
    {
        int f = 0, b = 0;
        DevSearch weak = G.search;
        const int d = bound_and_prune<NW>(T, S, weak, 0, R.row, n, f, b, 0, 0, best, rootc);
        vset<NW>(R.dir, 0, d);
    }
    store_row<NW>(G.ivm, id, 0, R.row);
    // path level 0: nothing fixed, every job free
    R.hf = 0;
    R.hb = 0;
    R.hr = 0;
    if (lane_id() < T.m)
        for (int j = 0; j < n; j++) R.hr += T.p[lane_id() * n + j];
    store_path<NW>(G.ivm, id, 0, R);
    NodeCounters nc = {0, 0, 0, 0, 0};
    const int mode = G.search.bound_mode;
    while (R.line < n - 2) {
        const int L = R.line;
        const int p = vget<NW>(R.pos, L);
        if (vget<NW>(R.row, p) < 0) break;             // pos below L are already 0
        vset<NW>(R.pj, L, vget<NW>(R.row, p));
        path_down<NW>(T, R, vget<NW>(R.row, p), vget<NW>(R.dir, L));
        int nr[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int idx = w * 32 + lane_id();
            int src = idx < p ? idx : idx + 1;
            if (src >= 32 * NW) src = 0;
            nr[w] = cell_job(vgather<NW>(R.row, src));
        }
#pragma unroll
        for (int w = 0; w < NW; w++) R.row[w] = nr[w];
        R.line = L + 1;
        store_path<NW>(G.ivm, id, R.line, R);
        const int f = front_count<NW>(R, R.line), b = R.line - f;
        partial_from_path(T, S, f, b, R.hf, R.hb, R.hr);
        const int prev = vget<NW>(R.dir, L);
        const int d = bound_and_prune<NW>(T, S, G.search, mode, R.row, n - R.line, f, b, R.line, prev, best, nc,
                                          true);
        vset<NW>(R.dir, R.line, d);
        store_row<NW>(G.ivm, id, R.line, R.row);
    }
    store_ivm<NW>(G.ivm, id, R);
    const bool alive = before_end<NW>(R.pos, R.end, n);
    if (lane_id() == 0) {
        atomicAdd(&G.ctl->simple_bounds, nc.simple);
        atomicAdd(&G.ctl->johnson_bounds, nc.johnson);
        atomicAdd(&G.ctl->root_simple, rootc.simple);
        atomicAdd(&G.ctl->jsweeps, nc.sweeps);
        atomicAdd(&G.ctl->jfree, nc.free_jobs);
        atomicAdd(&G.ctl->jchild, nc.swept_children);
        atomicAdd(&G.ctl->jdirect, nc.direct_children);
        atomicAdd(&G.ctl->jdirect_free, nc.direct_free);
        if (alive) {
            G.ivm.state[id] = IVM_ACTIVE;
            atomicAdd(&G.ctl->active, 1);
        }
    }
}

// Persistent explorer loop.  Warp w of a group serves explorers w, w+W, ...
// (W = warps of the group).  Runs until no explorer of the group holds work,
// or `budget_ns` of device time has passed, or `max_rounds` rounds.  VAR = 3
// is VAR 0 for boundingMode 2 with MinMin branching and no findAll (the
// default search), compiled in as constants; VAR = 0
// compiles the sortedDFS row sorts, the early Johnson exit and node sampling
// out of the hot loop; VAR = 1 follows each group's sortedDFS and
// earlyStopJohnson settings; VAR = 2 also records sampled nodes into the
// group's SampleBuf.
template <int NW, int VAR>
__global__ void __launch_bounds__(32 * PBB_WARPS_MAX, 1)
pbb_explore_kernel(const DevGroup* groups, const int* ngroups_d, int warps_per_cta, unsigned long long budget_ns,
                   int max_rounds, int select_budget)
{
    extern __shared__ __align__(16) unsigned char smem[];
    // the group count lives in device memory so that a captured launch
    // (fixed grid) serves any set of groups; CTAs past the last group exit
    const int ngroups = *ngroups_d;
    if (ngroups <= 0) return;
    const int gi = group_of_cta(groups, ngroups);
    const DevGroup G = groups[gi];
    if ((int)blockIdx.x >= G.first_cta + G.ctas) return;
    // each warp keeps its explorer's free-position masks when the launch
    // gave the room for them (the host sizes the launch with them if they fit)
    unsigned dyn_smem;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_smem));
    const int fm = G.inst.posj != nullptr &&
                   pbb_smem_plan(G.inst.n, G.inst.m, G.inst.Ppad, warps_per_cta, 1).total <= (int)dyn_smem;
    if (VAR == 3 && !fm) {
        // the fixed build relies on the masks; the host launches it only
        // with room for them
        if (threadIdx.x == 0) atomicOr(&G.ctl->status, PBB_ST_BADINPUT);
        return;
    }
    const SmemPlan sp = pbb_smem_plan(G.inst.n, G.inst.m, G.inst.Ppad, warps_per_cta, fm);
    CtaTables T;
    load_tables(G.inst, smem, sp, T);
    __syncthreads();
    const int wic = threadIdx.x >> 5;
    const WarpScratch S = warp_scratch(smem + sp.warp_off + wic * sp.warp_bytes, sp, T.n, T.m, T.Ppad);
    const int W = G.ctas * warps_per_cta;
    const int wid = (blockIdx.x - G.first_cta) * warps_per_cta + wic;
    const int mode = VAR == 3 ? 2 : G.search.bound_mode;
    const unsigned long long t0 = globaltimer_ns();

    WarpCounters C = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    Ivm<NW> R;
    int cached = -1;                   // explorer whose state is held in registers
    int since = 0;                     // nodes it decomposed since it got work or gave some away
    // explorers holding work once the first core_warps warps of every CTA
    // are busy (no more than that share of the explorers can be)
    const int core_warps = G.search.core_warps;
    const int core_active = min(core_warps * G.ctas, (int)((long long)G.ivm.count * core_warps / warps_per_cta));
    const bool core_warp = wic < core_warps;   // this warp always asks for work
    unsigned idle_ns = 500;            // back-off of a warp that found nothing to do
    int best = 0;
    if (lane_id() == 0) best = (int)(ld_volatile_u64(&G.ctl->best_key) >> 32);
    best = __shfl_sync(FULLMASK, best, 0);

    for (int round = 0; round < max_rounds; round++) {
        // loop control is decided by lane 0 and broadcast, so that the warp
        // never splits on values read at slightly different times
        int stop = 0, active = 0;
        if (lane_id() == 0) {
            active = ld_volatile_s32(&G.ctl->active);
            stop = active == 0 || globaltimer_ns() - t0 > budget_ns;
        }
        if (__shfl_sync(FULLMASK, stop, 0)) break;
        bool worked = false;
        bool busy = false;          // an explorer of this warp is active or offered
        int spare = -1;             // an idle explorer of this warp
        int id = cached;
        if (id >= 0) {
            // the explorer held in registers is ACTIVE, and only this warp can
            // change that: keep stepping it without polling
            busy = true;
        } else {
            for (int base = wid; base < G.ivm.count && id < 0; base += 32 * W) {
                // the states of up to 32 of this warp's explorers in one load
                // (lane j: explorer base + jW)
                const int mine = base + lane_id() * W;
                const int st_l = mine < G.ivm.count ? ld_volatile_s32(G.ivm.state + mine) : -1;
                const unsigned act = __ballot_sync(FULLMASK, st_l == IVM_ACTIVE);
                const unsigned idl = __ballot_sync(FULLMASK, st_l == IVM_IDLE);
                if (act || __any_sync(FULLMASK, st_l == IVM_QUEUED)) busy = true;
                if (spare < 0 && idl) spare = base + (__ffs(idl) - 1) * W;
                if (act) id = base + (__ffs(act) - 1) * W;
            }
            if (id >= 0) {
                int st = 0;
                if (lane_id() == 0) st = ld_acquire(G.ivm.state + id);   // orders the reads of its image
                st = __shfl_sync(FULLMASK, st, 0);
                if (st == IVM_ACTIVE) {
                    load_ivm<NW>(G.ivm, id, R);
                    cached = id;
                    since = 0;
                    if (S.fmask) fmask_build<NW>(T, S, R.row, T.n - R.line);
                } else {
                    id = -1;
                }
            }
        }
        if (id >= 0) {
            int gb = 0;
            if (lane_id() == 0) gb = (int)(ld_volatile_u64(&G.ctl->best_key) >> 32);
            gb = __shfl_sync(FULLMASK, gb, 0);
            if (gb < best) best = gb;
            // an explorer offers work once it has decomposed share_after nodes
            // since it got its interval or last split it: in a narrow tree,
            // splitting at every step hands out pieces that end before they
            // pay for the split, and keeps the donors splitting instead of
            // exploring
            if (since >= G.search.share_after && try_share<NW>(G, id, R) == 1) since = 0;
            const int r = select_node<NW, (VAR == 3)>(G, T, S, id, R, best, C, select_budget);
            if (r == 1) since++;
            if (r == 1)
                bound_current<NW, (VAR == 1 || VAR == 2), (VAR == 2), (VAR == 3 ? 3 : 0)>(G, T, S, id, R, mode, best, C);
            worked = true;
            if (C.decomposed >= (1u << 20)) flush_counters(G, C);
            if (r == 0) {
                // interval exhausted: leave the pool of busy explorers (the
                // registers need not go back: nobody resumes this interval)
                __syncwarp();
                cached = -1;
                if (lane_id() == 0) {
                    st_release(G.ivm.state + id, IVM_IDLE);
                    atomicSub(&G.ctl->active, 1);
                }
                __syncwarp();
            }
        }
        // A warp with nothing to do offers ONE of its idle explorers to the
        // donors: work is only split towards warps that would otherwise wait,
        // never towards a warp that is busy with another explorer.  The first
        // core_warps warps of every CTA always take part; the others join
        // once that many explorers per CTA hold work, so a narrow search is
        // not cut into pieces for warps it cannot feed, and a wide one still
        // gets every warp.
        const bool tier = core_warp || active >= core_active;
        if (!busy && spare >= 0 && lane_id() == 0 && tier) {
            st_release(G.ivm.state + spare, IVM_QUEUED);
            if (!queue_push(G, spare)) st_release(G.ivm.state + spare, IVM_IDLE);
        }
        __syncwarp();
        // idle warps back off (0.5 us doubling to 32 us): their polling
        // competes with the working warps for issue slots and L2
        if (!worked) {
            __nanosleep(idle_ns);
            idle_ns = idle_ns < 32000u ? 2 * idle_ns : idle_ns;
        } else {
            idle_ns = 500;
        }
    }
    if (cached >= 0) store_ivm<NW>(G.ivm, cached, R);
    flush_counters(G, C);
}

// Lower a group's incumbent to `ub` (bound found elsewhere, no permutation here).
__global__ void pbb_lower_ub_kernel(const DevGroup* groups, int g, int ub)
{
    atomicMin(&groups[g].ctl->best_key, ((unsigned long long)(unsigned)ub << 32) | 0xffffffffull);
}

// Children bounds of `count` nodes (warp per node): weak LBs of every free job
// appended at the front / back (bound_fsp_weak::boundChildren), Johnson LBs
// of the same children (bound_fsp_strong::bornes_calculer on the child), the
// node's own weak and Johnson LB, all indexed by job id (0 for fixed jobs).
template <int NW>
__global__ void pbb_bound_kernel(DevInstance I, int count, const int* sched, const int* l1s, const int* l2s,
                                 int* wb, int* we, int* sb, int* se, int* node_weak, int* node_strong,
                                 unsigned int* status, int warps_per_cta, int method, BoundExtra X)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const SmemPlan sp = pbb_smem_plan(I.n, I.m, I.Ppad, warps_per_cta);
    CtaTables T;
    load_tables(I, smem, sp, T);
    __syncthreads();
    const int wic = threadIdx.x >> 5;
    const WarpScratch S = warp_scratch(smem + sp.warp_off + wic * sp.warp_bytes, sp, T.n, T.m, T.Ppad);
    const int n = T.n;
    const int lane = lane_id();
    for (int node = blockIdx.x * warps_per_cta + wic; node < count; node += gridDim.x * warps_per_cta) {
        const int* s = sched + (size_t)node * n;
        const int l1 = l1s[node], l2 = l2s[node];
        const bool ok = l1 >= -1 && l2 <= n && l1 < l2;
        if (!ok) {
            if (lane == 0) atomicOr(status, PBB_ST_BADINPUT);
            continue;
        }
        const int f = l1 + 1, b = n - l2, k = l2 - l1 - 1;
        for (int i = lane; i < f; i += 32) S.fjob[i] = (unsigned char)s[i];
        for (int i = lane; i < b; i += 32) S.bjob[i] = (unsigned char)s[n - 1 - i];
        int row[NW];
        bool valid[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int idx = w * 32 + lane;
            valid[w] = idx < k;
            row[w] = valid[w] ? s[l1 + 1 + idx] : 0;
            if (valid[w]) S.rowj[idx] = (unsigned char)row[w];
        }
        __syncwarp();
        partial_schedule(T, S, f, b, k);
        int* owb = wb + (size_t)node * n;
        int* owe = we + (size_t)node * n;
        int* osb = sb + (size_t)node * n;
        int* ose = se + (size_t)node * n;
        for (int i = lane; i < n; i += 32) { owb[i] = 0; owe[i] = 0; osb[i] = 0; ose[i] = 0; }
        __syncwarp();
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (valid[w]) {
                owb[row[w]] = weak_front(T, S, row[w]);
                owe[row[w]] = weak_back(T, S, row[w]);
            }
        }
        if (X.prio_begin) {
            // idle-time priorities of the children (bound_fsp_weak.cpp:140-146, 172-178)
            int* opb = X.prio_begin + (size_t)node * n;
            int* ope = X.prio_end + (size_t)node * n;
            for (int i = lane; i < n; i += 32) { opb[i] = 0; ope[i] = 0; }
            __syncwarp();
#pragma unroll
            for (int w = 0; w < NW; w++) {
                if (valid[w]) {
                    opb[row[w]] = weak_front_idle(T, S, row[w]);
                    ope[row[w]] = weak_back_idle(T, S, row[w]);
                }
            }
        }
        if (X.strong_idle && lane == 0) {
            // couts[1] of bound_fsp_strong::bornes_calculer: idle time of the
            // fixed jobs' schedules (scheduleFront :457-478, scheduleBack
            // :490-509): 0 with nothing fixed in front for the front part, and
            // 0 altogether when nothing is fixed at the back; 0 as well with at
            // most one free job (the reference leaves it unset there)
            int idle = 0;
            if (k > 1 && b > 0) {
                int fr[PBB_MAX_M], bk[PBB_MAX_M];
                for (int q = 0; q < T.m; q++) { fr[q] = 0; bk[q] = 0; }
                for (int i = 0; i < f; i++) {
                    const int j = S.fjob[i];
                    fr[0] += T.p[j];
                    for (int q = 1; q < T.m; q++) {
                        idle += max(0, fr[q - 1] - fr[q]);
                        fr[q] = max(fr[q], fr[q - 1]) + T.p[q * n + j];
                    }
                }
                for (int i = 0; i < b; i++) {
                    const int j = S.bjob[i];
                    bk[T.m - 1] += T.p[(T.m - 1) * n + j];
                    for (int q = T.m - 2; q >= 0; q--) {
                        idle += max(0, bk[q + 1] - bk[q]);
                        bk[q] = max(bk[q], bk[q + 1]) + T.p[q * n + j];
                    }
                }
            }
            X.strong_idle[node] = idle;
        }
        const int wn = weak_node_lb(T, S);
        // node Johnson LB and children Johnson LBs
        int snode = 0;
        unsigned um[NW];
        job_mask<NW>(um, row, valid);
        const int x0 = vget<NW>(row, 0);
        const int x1 = vget<NW>(row, 1);
        if (k <= 1) {
            // at most one free job: the reference evaluates the full permutation
            int v = 0;
            if (lane == 0) {
                if (k == 1) {
                    v = makespan_split(T, S, x0, -1);
                } else {
                    for (int kk = 0; kk < T.m; kk++) v = max(v, S.frontZ[kk] + S.backZ[kk]);
                }
            }
            snode = __shfl_sync(FULLMASK, v, 0);
            // the one child on either side completes the permutation: its makespan
            if (k == 1 && lane == 0) { osb[x0] = snode; ose[x0] = snode; }
        } else {
            if (k == 2) {
                int mk = 0;
                if (lane < 2) mk = makespan_split(T, S, lane == 0 ? x0 : x1, lane == 0 ? x1 : x0);
                const int mxy = __shfl_sync(FULLMASK, mk, 0), myx = __shfl_sync(FULLMASK, mk, 1);
#pragma unroll
                for (int w = 0; w < NW; w++) {
                    if (valid[w]) {
                        osb[row[w]] = (row[w] == x0) ? mxy : myx;
                        ose[row[w]] = (row[w] == x0) ? myx : mxy;
                    }
                }
            }
            for (int i = lane; i < T.n; i += 32) { S.lbF[i] = 0; S.lbB[i] = 0; }
            __syncwarp();
            const bool kids = k >= 3;
            unsigned none[NW];
#pragma unroll
            for (int q = 0; q < NW; q++) none[q] = 0;
            if (kids) child_tables<NW>(T, S, row, k, true, um, true, um);
            int nl = 0;
            if (kids && method == 0) {
                johnson_children<NW>(T, S, um, true, um, true, um, &nl);
            } else if (kids && method == 2 && T.posj) {
                johnson_children<NW>(T, S, um, false, none, false, none, &nl);
                johnson_sweep_masked<NW>(T, S, k, true, um, true, um);
            } else {
                johnson_children<NW>(T, S, um, false, none, false, none, &nl);
                if (kids) {
                    // direct scans, two children at a time (front side, then back side)
                    int cjob[4] = {0, 0, 0, 0}, cside[4] = {0, 0, 0, 0};
                    int nc = 0;
                    for (int c = 0; c < 2 * k; c++) {
                        const int j = vget<NW>(row, c < k ? c : c - k);
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            if (nc == q) { cjob[q] = j; cside[q] = c < k ? 0 : 1; }
                        nc++;
                        if (nc == PBB_DIRECT_MAX || c == 2 * k - 1) {
                            if (T.posj) johnson_direct_masked<NW>(T, S, k, nc, cjob, cside, INT_MAX);
                            else johnson_direct<NW>(T, S, um, nc, cjob, cside);
                            nc = 0;
                        }
                    }
                }
            }
            snode = nl;
            if (kids) {
#pragma unroll
                for (int w = 0; w < NW; w++) {
                    if (valid[w]) {
                        osb[row[w]] = S.lbF[row[w]];
                        ose[row[w]] = S.lbB[row[w]];
                    }
                }
            }
        }
        if (lane == 0) {
            node_weak[node] = wn;
            node_strong[node] = snode;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// host-side launch wrappers (pbb_launch.h)
// ---------------------------------------------------------------------------
namespace pbbl {

int smem_bytes(int n, int m, int Ppad, int warps, int fmask) { return pbb_smem_plan(n, m, Ppad, warps, fmask).total; }

template <int NW, int VAR>
int explore_occupancy(int warps_per_cta, int smem)
{
    int blocks = 0;
    cudaFuncSetAttribute(pbb_explore_kernel<NW, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, pbb_explore_kernel<NW, VAR>, 32 * warps_per_cta, smem);
    return blocks;
}

int explore_ctas_per_sm(int nw, int warps_per_cta, int smem, int variant)
{
    if (nw == 1) {
        switch (variant) {
        case 1: return explore_occupancy<1, 1>(warps_per_cta, smem);
        case 2: return explore_occupancy<1, 2>(warps_per_cta, smem);
        case 3: return explore_occupancy<1, 3>(warps_per_cta, smem);
        default: return explore_occupancy<1, 0>(warps_per_cta, smem);
        }
    }
    switch (variant) {
    case 1: return explore_occupancy<2, 1>(warps_per_cta, smem);
    case 2: return explore_occupancy<2, 2>(warps_per_cta, smem);
    case 3: return explore_occupancy<2, 3>(warps_per_cta, smem);
    default: return explore_occupancy<2, 0>(warps_per_cta, smem);
    }
}

cudaError_t launch_reset(const DevGroup* groups, int ngroups, const int* ub, cudaStream_t st)
{
    dim3 grid(64, ngroups < 65535 ? ngroups : 65535);
    pbb_reset_kernel<<<grid, 256, 0, st>>>(groups, ngroups, ub);
    return cudaGetLastError();
}

cudaError_t launch_root(int nw, const DevGroup* groups, int ngroups, const int* roots, const int* ivals,
                        int root_stride, int smem, cudaStream_t st, int per_group, const int* ids)
{
    const int blocks = ngroups * per_group;
    if (nw == 1) {
        cudaFuncSetAttribute(pbb_root_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        pbb_root_kernel<1><<<blocks, 32, smem, st>>>(groups, ngroups, roots, ivals, root_stride, per_group, ids);
    } else {
        cudaFuncSetAttribute(pbb_root_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        pbb_root_kernel<2><<<blocks, 32, smem, st>>>(groups, ngroups, roots, ivals, root_stride, per_group, ids);
    }
    return cudaGetLastError();
}

cudaError_t launch_lower_ub(const DevGroup* groups, int g, int ub, cudaStream_t st)
{
    pbb_lower_ub_kernel<<<1, 1, 0, st>>>(groups, g, ub);
    return cudaGetLastError();
}

template <int NW, int VAR>
cudaError_t explore_launch(const DevGroup* groups, const int* ngroups_d, int ctas, int warps_per_cta, int smem,
                           unsigned long long budget_ns, int max_rounds, int select_budget, cudaStream_t st)
{
    cudaFuncSetAttribute(pbb_explore_kernel<NW, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    pbb_explore_kernel<NW, VAR><<<ctas, 32 * warps_per_cta, smem, st>>>(groups, ngroups_d, warps_per_cta, budget_ns,
                                                                         max_rounds, select_budget);
    return cudaGetLastError();
}

cudaError_t launch_explore(int nw, const DevGroup* groups, const int* ngroups_d, int ctas, int warps_per_cta, int smem,
                           unsigned long long budget_ns, int max_rounds, int select_budget, cudaStream_t st,
                           int variant)
{
#define PBB_EXPLORE(NW_, VAR_) \
    explore_launch<NW_, VAR_>(groups, ngroups_d, ctas, warps_per_cta, smem, budget_ns, max_rounds, select_budget, st)
    if (nw == 1) {
        switch (variant) {
        case 1: return PBB_EXPLORE(1, 1);
        case 2: return PBB_EXPLORE(1, 2);
        case 3: return PBB_EXPLORE(1, 3);
        default: return PBB_EXPLORE(1, 0);
        }
    }
    switch (variant) {
    case 1: return PBB_EXPLORE(2, 1);
    case 2: return PBB_EXPLORE(2, 2);
    case 3: return PBB_EXPLORE(2, 3);
    default: return PBB_EXPLORE(2, 0);
    }
#undef PBB_EXPLORE
}

cudaError_t launch_bound(int nw, const DevInstance& I, int count, const int* sched, const int* l1, const int* l2,
                         int* wb, int* we, int* sb, int* se, int* nweak, int* nstrong, unsigned int* status,
                         int ctas, int warps_per_cta, int smem, cudaStream_t st, int method, BoundExtra extra)
{
    if (nw == 1) {
        cudaFuncSetAttribute(pbb_bound_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        pbb_bound_kernel<1><<<ctas, 32 * warps_per_cta, smem, st>>>(I, count, sched, l1, l2, wb, we, sb, se, nweak,
                                                                     nstrong, status, warps_per_cta, method, extra);
    } else {
        cudaFuncSetAttribute(pbb_bound_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        pbb_bound_kernel<2><<<ctas, 32 * warps_per_cta, smem, st>>>(I, count, sched, l1, l2, wb, we, sb, se, nweak,
                                                                     nstrong, status, warps_per_cta, method, extra);
    }
    return cudaGetLastError();
}

}  // namespace pbbl
