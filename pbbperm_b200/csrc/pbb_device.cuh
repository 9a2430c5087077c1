// Warp-level device routines of the IVM flow-shop engine (sm_100a).
//
// One warp owns one IVM step at a time.  Per-level vectors (pos, end, dir,
// path job) and the current matrix row live in registers, element e of a
// vector at lane (e % 32), word (e / 32); the instance tables live in shared
// memory; the IVM matrix lives in HBM.  Everything is int32 and bit-exact
// with the reference bounds (bounds/src/bound_fsp_weak.cpp,
// bounds/src/bound_fsp_strong.cpp) and IVM navigation (multicore/src/ivm.cpp,
// ivm_bound.cpp, sequentialbb.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>
#include "pbb_types.h"

#define FULLMASK 0xffffffffu
#define NEG_INF (-(1 << 28))
// direct scans walk at most this many children together
#define PBB_DIRECT_MAX 4
// nodes with at most this many Johnson children use direct scans (by groups
// of PBB_DIRECT_MAX), more children use the max-plus sweeps
#ifndef PBB_DIRECT_LIMIT
#define PBB_DIRECT_LIMIT 4
#endif
// a lone child gets its own one-chain direct scan (instead of two chains, one
// repeating the other)
#ifndef PBB_DIRECT_ONE
#define PBB_DIRECT_ONE 1
#endif
// unroll factor of the loop that builds a pair's free-position mask
#ifndef PBB_FREEPOS_UNROLL
#define PBB_FREEPOS_UNROLL 1
#endif
// Loops over machines and over free jobs stay rolled: the explorer kernel is
// large and instruction-fetch bound, and unrolled copies of these loops cost
// more in fetch stalls than they save in loop overhead.
#define PBB_ROLLED _Pragma("unroll 1")
#define PBB_PRAGMA(x) _Pragma(#x)
#define PBB_UNROLL(n) PBB_PRAGMA(unroll n)

namespace pbb {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

// job stored in a cell, whatever its pruning flag (common/include/misc.h absolute())
__device__ __forceinline__ int cell_job(int v) { return v >= 0 ? v : -v - 1; }
// flagged form of a cell (misc.h negative())
__device__ __forceinline__ int cell_flag(int v) { return v < 0 ? v : -v - 1; }

// element `idx` (warp-uniform) of a lane-distributed vector
template <int NW>
__device__ __forceinline__ int vget(const int (&x)[NW], int idx)
{
    int src = x[0];
#pragma unroll
    for (int w = 1; w < NW; w++)
        if ((idx >> 5) == w) src = x[w];
    return __shfl_sync(FULLMASK, src, idx & 31);
}

// element `s` (per lane) of a lane-distributed vector
template <int NW>
__device__ __forceinline__ int vgather(const int (&x)[NW], int s)
{
    int r = 0;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        int t = __shfl_sync(FULLMASK, x[w], s & 31);
        if ((s >> 5) == w) r = t;
    }
    return r;
}

template <int NW>
__device__ __forceinline__ void vset(int (&x)[NW], int idx, int val)
{
    if (lane_id() == (idx & 31)) {
#pragma unroll
        for (int w = 0; w < NW; w++)
            if ((idx >> 5) == w) x[w] = val;
    }
}

// ivm.cpp:153-162 -- lexicographic pos <= end over the n levels
template <int NW>
__device__ __forceinline__ bool before_end(const int (&pos)[NW], const int (&end)[NW], int n)
{
#pragma unroll
    for (int w = 0; w < NW; w++) {
        int lv = w * 32 + lane_id();
        unsigned d = __ballot_sync(FULLMASK, lv < n && pos[w] != end[w]);
        if (d) {
            int f = __ffs(d) - 1;
            int pp = __shfl_sync(FULLMASK, pos[w], f);
            int ee = __shfl_sync(FULLMASK, end[w], f);
            return pp < ee;
        }
    }
    return true;
}

// first unpruned cell of the row at index >= from (and < k), or k
template <int NW>
__device__ __forceinline__ int next_open_cell(const int (&row)[NW], int from, int k)
{
#pragma unroll
    for (int w = 0; w < NW; w++) {
        int idx = w * 32 + lane_id();
        unsigned b = __ballot_sync(FULLMASK, idx >= from && idx < k && row[w] >= 0);
        if (b) return w * 32 + __ffs(b) - 1;
    }
    return k;
}

// ---------------------------------------------------------------------------
// shared-memory views
// ---------------------------------------------------------------------------
struct CtaTables {
    const unsigned long long* je;  // [n][Ppad]
    const int* p;                  // [m][n]
    const unsigned char* pm0;
    const unsigned char* pm1;
    const int* min_arr;
    const int* min_dep;
    const unsigned char* posj;     // [n][Ppad] or NULL
    int n, m, P, Ppad;
};

struct WarpScratch {
    int* lbF;     // [n] Johnson LB of front children, by job
    int* lbB;     // [n]
    int* frontZ;  // [32] heads of the front jobs (zero based)
    int* backZ;   // [32] tails of the back jobs (zero based)
    int* Fb;      // [32] front used by the bounds (earliest starts when no front job)
    int* Bb;      // [32] back used by the bounds (min run-outs when no back job)
    int* rem;     // [32] machine loads of the free jobs
    int* RB;      // [32] rem + Bb
    int* FR;      // [32] Fb + rem
    short* dF;    // [n][m] heads of front child u minus frontZ
    short* dB;    // [n][m] tails of back child u minus backZ
    unsigned char* fjob;  // [n] front jobs in schedule order
    unsigned char* bjob;  // [n] back jobs, last position first
    unsigned char* rowj;  // [n] free jobs (row order)
    // [Ppad] per machine pair, the Johnson positions of the free jobs of the
    // explorer this warp holds (bit t = position t), kept up to date by the
    // explorer as it moves; NULL outside the explorer or when it does not fit
    unsigned long long* fmask;
};

__device__ __forceinline__ WarpScratch warp_scratch(unsigned char* base, const SmemPlan& sp, int n, int m, int Ppad)
{
    WarpScratch s;
    s.fmask = nullptr;
    if (sp.fmask) {
        s.fmask = reinterpret_cast<unsigned long long*>(base);
        base += Ppad * 8;
    }
    int* ip = reinterpret_cast<int*>(base);
    s.lbF = ip; ip += n;
    s.lbB = ip; ip += n;
    s.frontZ = ip; ip += 32;
    s.backZ = ip; ip += 32;
    s.Fb = ip; ip += 32;
    s.Bb = ip; ip += 32;
    s.rem = ip; ip += 32;
    s.RB = ip; ip += 32;
    s.FR = ip; ip += 32;
    short* sp2 = reinterpret_cast<short*>(ip);
    s.dF = sp2; sp2 += n * m;
    s.dB = sp2; sp2 += n * m;
    unsigned char* bp = reinterpret_cast<unsigned char*>(sp2);
    s.fjob = bp; bp += n;
    s.bjob = bp; bp += n;
    s.rowj = bp;
    return s;
}

// ---------------------------------------------------------------------------
// partial schedules
// ---------------------------------------------------------------------------

// Heads of fjob[0..f) and tails of bjob[0..b), both from zero, one machine per
// lane, as a diagonal wavefront (bound_fsp_weak.cpp:62-107 restated).  Then
// the bound-side front/back: earliest starts when nothing is fixed in front,
// minimum run-outs when nothing is fixed at the back (:62-66, :86-90), and the
// loads of the free jobs (:110-122).
__device__ __forceinline__ void partial_schedule(const CtaTables& T, const WarpScratch& S, int f, int b, int k)
{
    const int lane = lane_id();
    const int n = T.n, m = T.m;
    int cf = 0, cb = 0;
    const int steps = (f > b ? f : b) + m - 1;
    const int ib0 = m - 1 - lane;
    for (int s = 0; s < steps; s++) {
        int upf = __shfl_up_sync(FULLMASK, cf, 1);
        int dnb = __shfl_down_sync(FULLMASK, cb, 1);
        if (lane == 0) upf = 0;
        if (lane == m - 1) dnb = 0;
        int i = s - lane;
        if (lane < m && i >= 0 && i < f) cf = max(cf, upf) + T.p[lane * n + S.fjob[i]];
        int ib = s - ib0;
        if (lane < m && ib >= 0 && ib < b) cb = max(cb, dnb) + T.p[lane * n + S.bjob[ib]];
    }
    if (lane < m) {
        // loads of the free jobs: sum the shorter of the free / fixed lists
        int r = 0;
        if (k <= n - k) {
            for (int i = 0; i < k; i++) r += T.p[lane * n + S.rowj[i]];
        } else {
            for (int j = 0; j < n; j++) r += T.p[lane * n + j];
            for (int i = 0; i < f; i++) r -= T.p[lane * n + S.fjob[i]];
            for (int i = 0; i < b; i++) r -= T.p[lane * n + S.bjob[i]];
        }
        int fb = (f == 0) ? T.min_arr[lane] : cf;
        int bb = (b == 0) ? T.min_dep[lane] : cb;
        S.frontZ[lane] = cf;
        S.backZ[lane] = cb;
        S.Fb[lane] = fb;
        S.Bb[lane] = bb;
        S.rem[lane] = r;
        S.RB[lane] = r + bb;
        S.FR[lane] = fb + r;
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// path partial schedule kept one machine per lane (lane k = machine k):
//   hf = heads of the front jobs, hb = tails of the back jobs (both zero
//   based), hr = loads of the free jobs.  Going down one level adds one job
//   to the front or to the back; both updates are exact max-plus scans.
// ---------------------------------------------------------------------------

// heads after appending job u: h_k = max(h_{k-1}, hf_k) + p_k(u), h_{-1} = 0,
// equal to P_k + max_{j<=k}(hf_j - P_{j-1}) with P the prefix sums of p(u)
// (heads are >= 0, so the h_{-1} term never wins)
__device__ __forceinline__ int append_front(const CtaTables& T, int hf, int u)
{
    const int lane = lane_id();
    const int pu = lane < T.m ? T.p[lane * T.n + u] : 0;
    int P = pu;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULLMASK, P, o);
        if (lane >= o) P += t;
    }
    int x = hf - (P - pu);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(FULLMASK, x, o);
        if (lane >= o) x = max(x, t);
    }
    return P + x;
}

// tails after putting job u first among the back jobs:
// t_k = max(t_{k+1}, hb_k) + p_k(u), t_m = 0, equal to
// Q_k + max_{j>=k}(hb_j - Q_{j+1}) with Q the suffix sums of p(u)
__device__ __forceinline__ int prepend_back(const CtaTables& T, int hb, int u)
{
    const int lane = lane_id();
    const bool on = lane < T.m;
    const int pu = on ? T.p[lane * T.n + u] : 0;
    int Q = pu;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_down_sync(FULLMASK, Q, o);
        if (lane + o < 32) Q += t;
    }
    int x = on ? hb - (Q - pu) : NEG_INF;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_down_sync(FULLMASK, x, o);
        if (lane + o < 32) x = max(x, t);
    }
    return Q + x;
}

// the bound-side arrays of the scratch from the path registers (what
// partial_schedule computes from the job lists)
__device__ __forceinline__ void partial_from_path(const CtaTables& T, const WarpScratch& S, int f, int b, int hf,
                                                  int hb, int hr)
{
    const int lane = lane_id();
    if (lane < T.m) {
        const int fb = (f == 0) ? T.min_arr[lane] : hf;
        const int bb = (b == 0) ? T.min_dep[lane] : hb;
        S.frontZ[lane] = hf;
        S.backZ[lane] = hb;
        S.Fb[lane] = fb;
        S.Bb[lane] = bb;
        S.rem[lane] = hr;
        S.RB[lane] = hr + bb;
        S.FR[lane] = fb + hr;
    }
    __syncwarp();
}

// weak node LB (bound_fsp_weak.cpp:289-311), read by every lane
__device__ __forceinline__ int weak_node_lb(const CtaTables& T, const WarpScratch& S)
{
    int t0 = S.Fb[0] + S.rem[0];
    int lb = t0 + S.Bb[0];
    PBB_ROLLED
    for (int k = 1; k < T.m; k++) {
        int t1 = max(S.FR[k], t0);
        lb = max(lb, t1 + S.Bb[k]);
        t0 = t1;
    }
    return lb;
}

// weak LB of child u appended at the front (bound_fsp_weak.cpp:134-161)
__device__ __forceinline__ int weak_front(const CtaTables& T, const WarpScratch& S, int u)
{
    const int n = T.n;
    int t0 = S.Fb[0] + T.p[u];
    int lb = S.Fb[0] + S.RB[0];
    PBB_ROLLED
    for (int k = 1; k < T.m; k++) {
        int t1 = max(S.Fb[k], t0);
        lb = max(lb, t1 + S.RB[k]);
        t0 = t1 + T.p[k * n + u];
    }
    return lb;
}

// weak LB of child u prepended at the back (bound_fsp_weak.cpp:164-191)
__device__ __forceinline__ int weak_back(const CtaTables& T, const WarpScratch& S, int u)
{
    const int n = T.n, m = T.m;
    int t0 = S.Bb[m - 1] + T.p[(m - 1) * n + u];
    int lb = S.FR[m - 1] + S.Bb[m - 1];
    PBB_ROLLED
    for (int k = m - 2; k >= 0; k--) {
        int t1 = max(t0, S.Bb[k]);
        lb = max(lb, S.FR[k] + t1);
        t0 = t1 + T.p[k * n + u];
    }
    return lb;
}

// idle-time priority of child u appended at the front: the sum over machines
// k >= 1 of |completion of u on k-1 - front_k| (bound_fsp_weak.cpp:140-146)
__device__ __forceinline__ int weak_front_idle(const CtaTables& T, const WarpScratch& S, int u)
{
    const int n = T.n;
    int t0 = S.Fb[0] + T.p[u];
    int pr = 0;
    PBB_ROLLED
    for (int k = 1; k < T.m; k++) {
        pr += abs(t0 - S.Fb[k]);
        t0 = max(S.Fb[k], t0) + T.p[k * n + u];
    }
    return pr;
}

// the same for child u prepended at the back (bound_fsp_weak.cpp:172-178)
__device__ __forceinline__ int weak_back_idle(const CtaTables& T, const WarpScratch& S, int u)
{
    const int n = T.n, m = T.m;
    int t0 = S.Bb[m - 1] + T.p[(m - 1) * n + u];
    int pr = 0;
    PBB_ROLLED
    for (int k = m - 2; k >= 0; k--) {
        pr += abs(t0 - S.Bb[k]);
        t0 = max(t0, S.Bb[k]) + T.p[k * n + u];
    }
    return pr;
}

// makespan of  front jobs + x + y + back jobs  (y < 0: front + x + back),
// as max over machines of head + tail at the split
__device__ __forceinline__ int makespan_split(const CtaTables& T, const WarpScratch& S, int x, int y)
{
    const int n = T.n;
    int h1 = 0, h2 = 0, best = 0;
    PBB_ROLLED
    for (int k = 0; k < T.m; k++) {
        h1 = max(h1, S.frontZ[k]) + T.p[k * n + x];
        int h = h1;
        if (y >= 0) { h2 = max(h2, h1) + T.p[k * n + y]; h = h2; }
        best = max(best, h + S.backZ[k]);
    }
    return best;
}

// ---------------------------------------------------------------------------
// Johnson two-machine bound of children (bound_fsp_strong.cpp:103-162 per child)
// ---------------------------------------------------------------------------
//
// For machine pair (a, b) with lag c and the free jobs U in Johnson order,
// the reference scans  t0 += a_j ; t1 = max(t1, t0 + c_j) + b_j  from
// (t0, t1) = (front[a], front[b]) and closes with max(t1 + back[b], t0 + back[a]).
// This map is max-plus linear: over a sequence it equals
//   t0' = t0 + A,   t1' = max(t1 + B, t0 + C),   C = max_s (Apre_s + c_s + Bsuf_s).
// Dropping the child's own job q from U gives
//   C_{-q} = max( max_{s<q} W_s - b_q , max_{s>q} W_s - a_q ),  W_s = Apre_s + c_s + Bsuf_s
// so one forward and one backward sweep per pair yield the LB of every child
// at once, exactly (integer max/+ only).  Lanes own machine pairs; the
// per-child maxima are merged with shared-memory atomicMax by job id.
//
// doF / doB select front / back children; sF / sB are job masks of the
// children to evaluate.  Results land in S.lbF / S.lbB (0 = not evaluated).
template <int NW>
__device__ __forceinline__ void johnson_children(const CtaTables& T, const WarpScratch& S,
                                                 const unsigned (&um)[NW], bool doF, const unsigned (&sF)[NW],
                                                 bool doB, const unsigned (&sB)[NW], int* node_lb)
{
    const int lane = lane_id();
    const int n = T.n, m = T.m;
    int nodeAcc = 0;
    for (int base = 0; base < T.P; base += 32) {
        const int i = base + lane;
        const bool act = i < T.P;
        const int m0 = act ? T.pm0[i] : 0;
        const int m1 = act ? T.pm1[i] : 0;
        const int Asum = S.rem[m0], Bsum = S.rem[m1];
        // front children: F = frontZ + dF[u], B = Bb
        const int cF1 = S.frontZ[m1] + Bsum + S.Bb[m1];
        const int cF2 = S.frontZ[m0] + S.Bb[m1];
        const int cF3 = S.frontZ[m0] + Asum + S.Bb[m0];
        // back children: F = Fb, B = backZ + dB[u]
        const int cB1 = S.Fb[m1] + Bsum + S.backZ[m1];
        const int cB2 = S.Fb[m0] + S.backZ[m1];
        const int cB3 = S.Fb[m0] + Asum + S.backZ[m0];
        const unsigned long long* col = T.je + i;
        int Apre = 0, Bpre = 0, PMx = NEG_INF;
        if (act) {
            for (int t = 0; t < n; t++) {
                const unsigned long long e = col[t * T.Ppad];
                const int u = JE_JOB(e);
                const unsigned bit = 1u << (u & 31);
                unsigned uw = um[0], fw = sF[0], bw = sB[0];
#pragma unroll
                for (int w = 1; w < NW; w++)
                    if ((u >> 5) == w) { uw = um[w]; fw = sF[w]; bw = sB[w]; }
                if (uw & bit) {
                    const int a = JE_A(e), b = JE_B(e), c = JE_C(e);
                    Apre += a;
                    const int W = Apre - Bpre + c + Bsum;
                    if (doF && (fw & bit)) {
                        const int d0 = S.dF[u * m + m0], d1 = S.dF[u * m + m1];
                        int v = max(cF1 + d1 - b, cF2 + d0 + PMx - b);
                        v = max(v, cF3 + d0 - a);
                        atomicMax(&S.lbF[u], v);
                    }
                    if (doB && (bw & bit)) {
                        const int d0 = S.dB[u * m + m0], d1 = S.dB[u * m + m1];
                        int v = max(cB1 - b, cB2 + PMx - b) + d1;
                        v = max(v, cB3 - a + d0);
                        atomicMax(&S.lbB[u], v);
                    }
                    PMx = max(PMx, W);
                    Bpre += b;
                }
            }
            if (node_lb) {
                // the node itself (nothing removed): bornes_calculer of the node
                int v = max(S.Fb[m1] + Bsum + S.Bb[m1], S.Fb[m0] + PMx + S.Bb[m1]);
                v = max(v, S.Fb[m0] + Asum + S.Bb[m0]);
                nodeAcc = max(nodeAcc, v);
            }
            int Asuf = 0, Bsuf = 0, SMx = NEG_INF;
            for (int t = n - 1; t >= 0; t--) {
                const unsigned long long e = col[t * T.Ppad];
                const int u = JE_JOB(e);
                const unsigned bit = 1u << (u & 31);
                unsigned uw = um[0], fw = sF[0], bw = sB[0];
#pragma unroll
                for (int w = 1; w < NW; w++)
                    if ((u >> 5) == w) { uw = um[w]; fw = sF[w]; bw = sB[w]; }
                if (uw & bit) {
                    const int a = JE_A(e), b = JE_B(e), c = JE_C(e);
                    if (doF && (fw & bit)) {
                        const int d0 = S.dF[u * m + m0];
                        atomicMax(&S.lbF[u], cF2 + d0 + SMx - a);
                    }
                    if (doB && (bw & bit)) {
                        const int d1 = S.dB[u * m + m1];
                        atomicMax(&S.lbB[u], cB2 + SMx - a + d1);
                    }
                    Bsuf += b;
                    SMx = max(SMx, Asum - Asuf + c + Bsuf);
                    Asuf += a;
                }
            }
        }
    }
    if (node_lb) {
        for (int o = 16; o; o >>= 1) nodeAcc = max(nodeAcc, __shfl_xor_sync(FULLMASK, nodeAcc, o));
        *node_lb = nodeAcc;
    }
    __syncwarp();
}

// Johnson LB of a few children by direct scans (bound_fsp_strong.cpp:76-100
// run per child): lanes own (machine pair, child) combinations, each scans the
// pair's Johnson order over the free jobs minus the child's own job, with the
// recurrence predicated instead of branched, and merges its pair maximum with
// one shared-memory atomicMax.  Cheaper than the two sweeps of
// johnson_children when only one to three children are evaluated.
// cjob/cside: the children's jobs and sides (0 front, 1 back), nc <= 4.
template <int NW>
__device__ __forceinline__ void johnson_direct(const CtaTables& T, const WarpScratch& S, const unsigned (&um)[NW],
                                               int nc, const int (&cjob)[4], const int (&cside)[4])
{
    const int lane = lane_id();
    const int n = T.n, m = T.m, P = T.P;
    const unsigned long long free_all =
        (NW > 1 ? ((unsigned long long)um[NW > 1 ? 1 : 0] << 32) : 0ull) | (unsigned long long)um[0];
    const int combos = P * nc;
    for (int base = 0; base < combos; base += 32) {
        const int q = base + lane;
        if (q < combos) {
            int ci = 0, i = q;
            while (i >= P) { i -= P; ci++; }
            int u = cjob[0], side = cside[0];
#pragma unroll
            for (int c = 1; c < 4; c++)
                if (ci == c) { u = cjob[c]; side = cside[c]; }
            const int m0 = T.pm0[i], m1 = T.pm1[i];
            int t0, t1, B0, B1;
            if (side == 0) {
                t0 = S.frontZ[m0] + S.dF[u * m + m0];
                t1 = S.frontZ[m1] + S.dF[u * m + m1];
                B0 = S.Bb[m0];
                B1 = S.Bb[m1];
            } else {
                t0 = S.Fb[m0];
                t1 = S.Fb[m1];
                B0 = S.backZ[m0] + S.dB[u * m + m0];
                B1 = S.backZ[m1] + S.dB[u * m + m1];
            }
            const unsigned long long fm = free_all & ~(1ull << u);
            const unsigned long long* col = T.je + i;
#pragma unroll 2
            for (int t = 0; t < n; t++) {
                const unsigned long long e = col[t * T.Ppad];
                const bool fr = (fm >> JE_JOB(e)) & 1ull;
                const int t0n = t0 + JE_A(e);
                const int t1n = max(t1, t0n + JE_C(e)) + JE_B(e);
                t0 = fr ? t0n : t0;
                t1 = fr ? t1n : t1;
            }
            atomicMax(side ? &S.lbB[u] : &S.lbF[u], max(t1 + B1, t0 + B0));
        }
    }
    __syncwarp();
}

// Johnson positions (for the lane's pair i) holding a free job, as a 64-bit
// mask built from the inverse Johnson order T.posj: scans then visit only the
// k free positions instead of all n.
// Position masks over a pair's Johnson order: 32 bits are enough for rows of
// one word (n <= 32), and cheaper to walk than 64.
template <int NW>
struct PosMask {
    typedef unsigned long long type;
};
template <>
struct PosMask<1> {
    typedef unsigned type;
};

__device__ __forceinline__ int low_pos(unsigned m) { return __ffs(m) - 1; }
__device__ __forceinline__ int low_pos(unsigned long long m) { return __ffsll((long long)m) - 1; }
__device__ __forceinline__ int high_pos(unsigned m) { return 31 - __clz(m); }
__device__ __forceinline__ int high_pos(unsigned long long m) { return 63 - __clzll((long long)m); }

// Johnson positions of the free jobs (rowj[0..k)) for machine pair i, as a mask
template <int NW>
__device__ __forceinline__ typename PosMask<NW>::type free_positions(const CtaTables& T, const WarpScratch& S, int k,
                                                                     int i)
{
    typedef typename PosMask<NW>::type M;
    const unsigned char* col = T.posj + i;
    M pm = 0;
    PBB_UNROLL(PBB_FREEPOS_UNROLL)
    for (int q = 0; q < k; q++) pm |= (M)1 << col[S.rowj[q] * T.Ppad];
    return pm;
}

// The free-position masks of the explorer a warp holds (S.fmask, explorer
// only): built from the row at its line when the warp takes the explorer,
// then kept exact by flipping one bit per machine pair as it moves: going
// down removes the chosen job, going up puts back the job of the level it
// returns to.  The bound then reads one word per pair instead of rebuilding
// the mask from the k free jobs at every node.
template <int NW>
__device__ __forceinline__ void fmask_build(const CtaTables& T, const WarpScratch& S, const int (&row)[NW], int k)
{
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int idx = w * 32 + lane_id();
        if (idx < k) S.rowj[idx] = (unsigned char)cell_job(row[w]);
    }
    __syncwarp();
    for (int i = lane_id(); i < T.P; i += 32) S.fmask[i] = (unsigned long long)free_positions<NW>(T, S, k, i);
    __syncwarp();
}

__device__ __forceinline__ void fmask_flip(const CtaTables& T, const WarpScratch& S, int u)
{
    const unsigned char* col = T.posj + u * T.Ppad;
    for (int i = lane_id(); i < T.P; i += 32) S.fmask[i] ^= 1ull << col[i];
    __syncwarp();
}

// the free-position mask of pair i for the node being bounded (FM: the
// warp's masks are known to be there)
template <int NW, int FM = 0>
__device__ __forceinline__ typename PosMask<NW>::type node_positions(const CtaTables& T, const WarpScratch& S, int k,
                                                                     int i)
{
    typedef typename PosMask<NW>::type M;
    if (FM) return (M)S.fmask[i];
    return S.fmask ? (M)S.fmask[i] : free_positions<NW>(T, S, k, i);
}

// Scan start of child u on pair (m0, m1): front child = heads of front + u,
// remaining back as is; back child = heads of front, tails of u + back.
__device__ __forceinline__ void direct_start(const CtaTables& T, const WarpScratch& S, int u, int side, int m0, int m1,
                                             int& t0, int& t1, int& B0, int& B1)
{
    const int m = T.m;
    if (side == 0) {
        t0 = S.frontZ[m0] + S.dF[u * m + m0];
        t1 = S.frontZ[m1] + S.dF[u * m + m1];
        B0 = S.Bb[m0];
        B1 = S.Bb[m1];
    } else {
        t0 = S.Fb[m0];
        t1 = S.Fb[m1];
        B0 = S.backZ[m0] + S.dB[u * m + m0];
        B1 = S.backZ[m1] + S.dB[u * m + m1];
    }
}

// johnson_direct over the free positions only (needs T.posj), one lane per
// machine pair: the pair's free-position mask is built once and the scans of
// up to C children walk it together, each skipping its own job by a select, so
// that the loop body has no branch (cutting the walk at the own positions
// instead made the lanes of a warp diverge and ran slower).  Chains past the
// child count repeat the first child and are not stored.  Child maxima over
// the pairs are taken with one warp reduction per pass.  Early exit
// (earlyStopJohnson, bound_fsp_strong.cpp:154-158): once every child's
// running maximum exceeds `stop` the remaining passes are skipped; such a
// child is pruned whatever its remaining pairs give, so only the value of a
// pruned child changes (INT_MAX = no early exit).
template <int C, int NW, int FM = 0>
__device__ __forceinline__ void johnson_direct_chains(const CtaTables& T, const WarpScratch& S, int k, int nc,
                                                      const int (&cjob)[4], const int (&cside)[4], int stop)
{
    typedef typename PosMask<NW>::type M;
    const int lane = lane_id();
    const int P = T.P;
    int u[C], sd[C], acc[C];
#pragma unroll
    for (int c = 0; c < C; c++) {
        u[c] = c < nc ? cjob[c] : cjob[0];
        sd[c] = c < nc ? cside[c] : cside[0];
        acc[c] = 0;                    // child LBs are positive
    }
    for (int base = 0; base < P; base += 32) {
        const int i = base + lane;
        int v[C];
#pragma unroll
        for (int c = 0; c < C; c++) v[c] = 0;
        if (i < P) {
            const int m0 = T.pm0[i], m1 = T.pm1[i];
            int t0[C], t1[C], B0[C], B1[C], px[C];
#pragma unroll
            for (int c = 0; c < C; c++) {
                direct_start(T, S, u[c], sd[c], m0, m1, t0[c], t1[c], B0[c], B1[c]);
                px[c] = T.posj[u[c] * T.Ppad + i];
            }
            M pm = node_positions<NW, FM>(T, S, k, i);
            const unsigned long long* col = T.je + i;
            while (pm) {
                const int t = low_pos(pm);
                pm &= pm - 1;
                const unsigned long long e = col[t * T.Ppad];
                const int a = JE_A(e), bb = JE_B(e), cc = JE_C(e);
#pragma unroll
                for (int c = 0; c < C; c++) {
                    t0[c] += t != px[c] ? a : 0;
                    const int nx = max(t1[c], t0[c] + cc) + bb;
                    t1[c] = t != px[c] ? nx : t1[c];
                }
            }
#pragma unroll
            for (int c = 0; c < C; c++) v[c] = max(t1[c] + B1[c], t0[c] + B0[c]);
        }
        bool over = true;
#pragma unroll
        for (int c = 0; c < C; c++) {
            acc[c] = max(acc[c], __reduce_max_sync(FULLMASK, v[c]));
            over = over && acc[c] > stop;
        }
        if (over) break;
    }
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < C; c++) {
            if (c < nc) {
                int* d = sd[c] ? &S.lbB[u[c]] : &S.lbF[u[c]];
                *d = max(*d, acc[c]);
            }
        }
    }
    __syncwarp();
}

template <int NW, int FM = 0>
__device__ __forceinline__ void johnson_direct_masked(const CtaTables& T, const WarpScratch& S, int k, int nc,
                                                      const int (&cjob)[4], const int (&cside)[4], int stop)
{
    static_assert(PBB_DIRECT_MAX <= 4, "direct scans walk at most four children together");
    if (nc <= 0) return;
#if PBB_DIRECT_ONE
    if (nc == 1) johnson_direct_chains<1, NW, FM>(T, S, k, nc, cjob, cside, stop);
    else
#endif
    if (nc <= 2) johnson_direct_chains<2, NW, FM>(T, S, k, nc, cjob, cside, stop);
    else johnson_direct_chains<4, NW, FM>(T, S, k, nc, cjob, cside, stop);
}

// johnson_children (forward + backward max-plus sweeps) over the free
// positions only (needs T.posj); same results, O(P k) instead of O(P n).
template <int NW, int FM = 0>
__device__ __forceinline__ void johnson_sweep_masked(const CtaTables& T, const WarpScratch& S, int k,
                                                     bool doF,
                                                     const unsigned (&sF)[NW], bool doB, const unsigned (&sB)[NW])
{
    const int lane = lane_id();
    const int m = T.m;
    for (int base = 0; base < T.P; base += 32) {
        const int i = base + lane;
        if (i < T.P) {
            const int m0 = T.pm0[i], m1 = T.pm1[i];
            const int Asum = S.rem[m0], Bsum = S.rem[m1];
            const int cF1 = S.frontZ[m1] + Bsum + S.Bb[m1];
            const int cF2 = S.frontZ[m0] + S.Bb[m1];
            const int cF3 = S.frontZ[m0] + Asum + S.Bb[m0];
            const int cB1 = S.Fb[m1] + Bsum + S.backZ[m1];
            const int cB2 = S.Fb[m0] + S.backZ[m1];
            const int cB3 = S.Fb[m0] + Asum + S.backZ[m0];
            const unsigned long long* col = T.je + i;
            typedef typename PosMask<NW>::type M;
            const M pm = node_positions<NW, FM>(T, S, k, i);
            int Apre = 0, Bpre = 0, PMx = NEG_INF;
            M fwd = pm;
            while (fwd) {
                const int t = low_pos(fwd);
                fwd &= fwd - 1;
                const unsigned long long e = col[t * T.Ppad];
                const int u = JE_JOB(e);
                const unsigned bit = 1u << (u & 31);
                unsigned fw = sF[0], bw = sB[0];
#pragma unroll
                for (int w = 1; w < NW; w++)
                    if ((u >> 5) == w) { fw = sF[w]; bw = sB[w]; }
                const int a = JE_A(e), b = JE_B(e), c = JE_C(e);
                Apre += a;
                const int W = Apre - Bpre + c + Bsum;
                if (doF && (fw & bit)) {
                    const int d0 = S.dF[u * m + m0], d1 = S.dF[u * m + m1];
                    atomicMax(&S.lbF[u], max(max(cF1 + d1 - b, cF2 + d0 + PMx - b), cF3 + d0 - a));
                }
                if (doB && (bw & bit)) {
                    const int d0 = S.dB[u * m + m0], d1 = S.dB[u * m + m1];
                    atomicMax(&S.lbB[u], max(max(cB1 - b, cB2 + PMx - b) + d1, cB3 - a + d0));
                }
                PMx = max(PMx, W);
                Bpre += b;
            }
            int Asuf = 0, Bsuf = 0, SMx = NEG_INF;
            M r = pm;
            while (r) {
                const int t = high_pos(r);
                r &= ~((M)1 << t);
                const unsigned long long e = col[t * T.Ppad];
                const int u = JE_JOB(e);
                const unsigned bit = 1u << (u & 31);
                unsigned fw = sF[0], bw = sB[0];
#pragma unroll
                for (int w = 1; w < NW; w++)
                    if ((u >> 5) == w) { fw = sF[w]; bw = sB[w]; }
                const int a = JE_A(e), b = JE_B(e), c = JE_C(e);
                if (doF && (fw & bit)) atomicMax(&S.lbF[u], cF2 + S.dF[u * m + m0] + SMx - a);
                if (doB && (bw & bit)) atomicMax(&S.lbB[u], cB2 + SMx - a + S.dB[u * m + m1]);
                Bsuf += b;
                SMx = max(SMx, Asum - Asuf + c + Bsuf);
                Asuf += a;
            }
        }
    }
    __syncwarp();
}

// Per-child head/tail deltas used by johnson_children (front child u: heads of
// front + u; back child u: tails of u + back).  Lane per free cell.
template <int NW>
__device__ __forceinline__ void child_tables(const CtaTables& T, const WarpScratch& S, const int (&row)[NW], int k,
                                             bool doF, const unsigned (&sF)[NW], bool doB, const unsigned (&sB)[NW])
{
    const int n = T.n, m = T.m;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        const int idx = w * 32 + lane_id();
        if (idx < k) {
            const int u = row[w];
            const unsigned bit = 1u << (u & 31);
            unsigned fw = sF[0], bw = sB[0];
#pragma unroll
            for (int q = 1; q < NW; q++)
                if ((u >> 5) == q) { fw = sF[q]; bw = sB[q]; }
            if (doF && (fw & bit)) {
                int h = 0;
                PBB_ROLLED
                for (int kk = 0; kk < m; kk++) {
                    const int z = S.frontZ[kk];
                    h = max(h, z) + T.p[kk * n + u];
                    S.dF[u * m + kk] = (short)(h - z);
                }
            }
            if (doB && (bw & bit)) {
                int t = 0;
                PBB_ROLLED
                for (int kk = m - 1; kk >= 0; kk--) {
                    const int z = S.backZ[kk];
                    t = max(t, z) + T.p[kk * n + u];
                    S.dB[u * m + kk] = (short)(t - z);
                }
            }
        }
    }
    __syncwarp();
}

// job bitmask of the lanes' cells where pred holds
template <int NW>
__device__ __forceinline__ void job_mask(unsigned (&out)[NW], const int (&row)[NW], const bool (&pred)[NW])
{
#pragma unroll
    for (int q = 0; q < NW; q++) {
        unsigned v = 0;
#pragma unroll
        for (int w = 0; w < NW; w++)
            if (pred[w] && ((row[w] >> 5) == q)) v |= 1u << (row[w] & 31);
        out[q] = __reduce_or_sync(FULLMASK, v);
    }
}

// Branching rule (ivm_bound.cpp:413-560, CPU numbering), evaluated over the
// free children only: fixed jobs have cost 0 on both sides and contribute
// nothing to any rule.  Returns 0 = FRONT, 1 = BACK.
template <int NW>
__device__ __forceinline__ int choose_dir(int rule, int line, int ub, const int (&cb)[NW], const int (&ce)[NW],
                                          const bool (&valid)[NW])
{
    switch (rule) {
    case -3: return (line & 1) ? 1 : 0;
    case -2: return 1;
    case -1: return 0;
    case 1: {
        int s = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) if (valid[w]) s += cb[w] - ce[w];
        s = __reduce_add_sync(FULLMASK, s);
        return s < 0 ? 1 : 0;
    }
    case 2: {
        int elim = 0, s = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (!valid[w]) continue;
            if (cb[w] >= ub) elim++; else s += cb[w];
            if (ce[w] >= ub) elim--; else s -= ce[w];
        }
        elim = __reduce_add_sync(FULLMASK, elim);
        s = __reduce_add_sync(FULLMASK, s);
        if (elim > 0) return 0;
        if (elim < 0) return 1;
        return s < 0 ? 1 : 0;
    }
    default: {   // 3: MinMin, ties broken by the eliminated count
        unsigned mn = 0x7fffffffu;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (!valid[w]) continue;
            if (cb[w] > 0) mn = min(mn, (unsigned)cb[w]);
            if (ce[w] > 0) mn = min(mn, (unsigned)ce[w]);
        }
        mn = __reduce_min_sync(FULLMASK, mn);
        int cnt = 0, elim = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (!valid[w]) continue;
            if ((unsigned)cb[w] == mn) cnt++;
            if ((unsigned)ce[w] == mn) cnt--;
            if (cb[w] >= ub) elim++;
            if (ce[w] >= ub) elim--;
        }
        cnt = __reduce_add_sync(FULLMASK, cnt);
        elim = __reduce_add_sync(FULLMASK, elim);
        if (cnt > 0) return 1;
        if (cnt < 0) return 0;
        return elim > 0 ? 0 : 1;
    }
    }
}

struct NodeCounters {
    unsigned simple, johnson;
    unsigned sweeps, free_jobs, swept_children, direct_children, direct_free;
};

// Bound the children of the node whose free jobs are `row[0..k)` (front and
// back lists already in S.fjob / S.bjob, f and b long), choose the branching
// side and prune the row in place (ivm_bound.cpp weak/strong/mixedBoundPrune
// :650-676 -> chooseChildrenSet, prune :611-646 with sortedDFS = 0).
// Stable sort of a row's k cells (k <= 64; lane l holds cells l and 32 + l) by
// key, written to out[0..k): a cell's place = cells with a smaller key plus
// earlier cells with the same key, the order gnomeSortByKeyInc and
// gnomeSortByKeysInc (misc.h:33-65) leave.  Keys are 64-bit so that a
// (cost, priority) pair sorts as one.  Called by all 32 lanes.
__device__ __noinline__ void sort_cells(unsigned char* out, int k, unsigned long long key0, unsigned long long key1,
                                        int cell0, int cell1)
{
    const int lane = lane_id();
    int r0 = 0, r1 = 0;
    PBB_ROLLED
    for (int j = 0; j < k; j++) {
        const unsigned long long kj = __shfl_sync(FULLMASK, j < 32 ? key0 : key1, j & 31);
        r0 += (kj < key0 || (kj == key0 && j < lane)) ? 1 : 0;
        r1 += (kj < key1 || (kj == key1 && j < lane + 32)) ? 1 : 0;
    }
    if (lane < k) out[r0] = (unsigned char)(signed char)cell0;
    if (lane + 32 < k) out[r1] = (unsigned char)(signed char)cell1;
    __syncwarp();
}

// Returns the side chosen for this level.  SAMPLE = 1 with `rec` set writes
// the children's bounds, as computed and before pruning, into a node record
// (SampleBuf layout: schedule at rec + PBB_SAMPLE_HDR, then four arrays of n).
// RULE != 0 fixes the branching rule at compile time (the caller then passes
// a constant mode too), so the hot explorer carries no code for the others.
template <int NW, int SORT = 1, int SAMPLE = 0, int RULE = 0>
__device__ __forceinline__ int bound_and_prune(const CtaTables& T, const WarpScratch& S, const DevSearch& srch,
                                               int mode, int (&row)[NW], int k, int f, int b, int line,
                                               int prev_dir, int best, NodeCounters& cnt, bool partial_ready = false,
                                               int* rec = nullptr)
{
    const int lane = lane_id();
    bool valid[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) valid[w] = (w * 32 + lane) < k;
#pragma unroll
    for (int w = 0; w < NW; w++)
        if (valid[w]) S.rowj[w * 32 + lane] = (unsigned char)row[w];
    __syncwarp();
    if (!partial_ready) partial_schedule(T, S, f, b, k);

    // the fixed build (RULE != 0) serves searches without findAll, with the
    // position tables present and the warp's free-position masks kept
    const bool both = (RULE ? RULE : srch.branch_mode) > 0;
    const bool fa = RULE ? false : srch.find_all != 0;
    const bool masked = RULE || T.posj;
    int cbw[NW], cew[NW], cbs[NW], ces[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) { cbw[w] = 0; cew[w] = 0; cbs[w] = 0; ces[w] = 0; }

    int dir;
    if (mode != 1) {
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (valid[w]) {
                cbw[w] = weak_front(T, S, row[w]);
                if (both) cew[w] = weak_back(T, S, row[w]);
            }
        }
        cnt.simple += both ? 2 * k : k;
        dir = choose_dir<NW>(RULE ? RULE : srch.branch_mode, line, best, cbw, cew, valid);
    }

    if (mode != 0) {
        bool doF = (mode == 1) || dir == 0;
        bool doB = (mode == 1) || dir == 1;
        bool pF[NW], pB[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            // mode 2 evaluates only the children the weak bound keeps (ivm_bound.cpp:168)
            bool keepF = (mode == 1) || !(fa ? cbw[w] > best : cbw[w] >= best);
            bool keepB = (mode == 1) || !(fa ? cew[w] > best : cew[w] >= best);
            pF[w] = valid[w] && doF && keepF;
            pB[w] = valid[w] && doB && keepB;
        }
        unsigned sF[NW], sB[NW], um[NW];
        job_mask<NW>(sF, row, pF);
        job_mask<NW>(sB, row, pB);
        job_mask<NW>(um, row, valid);
        int nF = 0, nB = 0;
#pragma unroll
        for (int q = 0; q < NW; q++) { nF += __popc(sF[q]); nB += __popc(sB[q]); }
        cnt.johnson += nF + nB;
        if (nF + nB > 0) {
            if (k <= 2) {
                // each child has at most one free job left: exact makespan
                // (bound_fsp_strong.cpp:543-546)
                const int x = vget<NW>(row, 0);
                const int y = k == 2 ? vget<NW>(row, 1) : -1;
                int mk = 0;
                if (lane < 2) mk = makespan_split(T, S, lane == 0 ? x : y, lane == 0 ? y : x);
                const int mxy = __shfl_sync(FULLMASK, mk, 0);
                const int myx = __shfl_sync(FULLMASK, mk, 1);
#pragma unroll
                for (int w = 0; w < NW; w++) {
                    if (pF[w]) cbs[w] = (row[w] == x) ? mxy : myx;
                    if (pB[w]) ces[w] = (row[w] == x) ? myx : mxy;
                }
            } else {
#pragma unroll
                for (int w = 0; w < NW; w++) {
                    if (w * 32 + lane < T.n) { S.lbF[w * 32 + lane] = 0; S.lbB[w * 32 + lane] = 0; }
                }
                child_tables<NW>(T, S, row, k, nF > 0, sF, nB > 0, sB);
                if (nF + nB <= PBB_DIRECT_LIMIT) {
#if PBB_DIRECT_LIMIT > PBB_DIRECT_MAX
                    // list the children (front side first, job order), then
                    // scan them by groups of at most PBB_DIRECT_MAX
                    int list[PBB_DIRECT_LIMIT];
                    int nc = 0;
#pragma unroll
                    for (int side = 0; side < 2; side++) {
#pragma unroll
                        for (int q = 0; q < NW; q++) {
                            unsigned msk = side ? sB[q] : sF[q];
                            while (msk) {
                                const int j = q * 32 + __ffs(msk) - 1;
                                msk &= msk - 1;
#pragma unroll
                                for (int c = 0; c < PBB_DIRECT_LIMIT; c++)
                                    if (nc == c) list[c] = j | (side << 8);
                                nc++;
                            }
                        }
                    }
                    // the early exit lives in the runtime-options build only (SORT = 1):
                    // the default explorer passes a constant and keeps no trace of it
                    const int stop = (SORT && srch.early_stop) ? best : INT_MAX;
                    PBB_ROLLED
                    for (int g = 0; g < nc; g += PBB_DIRECT_MAX) {
                        int cjob[4] = {0, 0, 0, 0}, cside[4] = {0, 0, 0, 0};
#pragma unroll
                        for (int c = 0; c < 4; c++) {
#pragma unroll
                            for (int e = 0; e < PBB_DIRECT_LIMIT; e++)
                                if (e == g + c) { cjob[c] = list[e] & 0xff; cside[c] = list[e] >> 8; }
                        }
                        const int gn = min(nc - g, PBB_DIRECT_MAX);
                        if (T.posj) johnson_direct_masked<NW>(T, S, k, gn, cjob, cside, stop);
                        else johnson_direct<NW>(T, S, um, gn, cjob, cside);
                    }
#else
                    // list the children (front side first, job order)
                    int cjob[4] = {0, 0, 0, 0}, cside[4] = {0, 0, 0, 0};
                    int nc = 0;
#pragma unroll
                    for (int side = 0; side < 2; side++) {
#pragma unroll
                        for (int q = 0; q < NW; q++) {
                            unsigned msk = side ? sB[q] : sF[q];
                            while (msk) {
                                const int j = q * 32 + __ffs(msk) - 1;
                                msk &= msk - 1;
#pragma unroll
                                for (int c = 0; c < 4; c++)
                                    if (nc == c) { cjob[c] = j; cside[c] = side; }
                                nc++;
                            }
                        }
                    }
                    // early exit: in the runtime-options build (SORT = 1) when
                    // earlyStopJohnson asks for it; in the default search's build
                    // (RULE != 0) always -- it only changes the values of
                    // children that are pruned anyway, which that build never
                    // reports; the general hot build keeps no trace of it
                    const int stop = RULE ? best : ((SORT && srch.early_stop) ? best : INT_MAX);
                    if (masked) johnson_direct_masked<NW, (RULE != 0)>(T, S, k, nc, cjob, cside, stop);
                    else johnson_direct<NW>(T, S, um, nc, cjob, cside);
#endif
                    cnt.direct_children += nc;
                    cnt.direct_free += (unsigned)(nc * k);
                } else {
                    if (masked) johnson_sweep_masked<NW, (RULE != 0)>(T, S, k, nF > 0, sF, nB > 0, sB);
                    else johnson_children<NW>(T, S, um, nF > 0, sF, nB > 0, sB, nullptr);
                    cnt.sweeps++;
                    cnt.free_jobs += k;
                    cnt.swept_children += nF + nB;
                }
#pragma unroll
                for (int w = 0; w < NW; w++) {
                    if (pF[w]) cbs[w] = S.lbF[row[w]];
                    if (pB[w]) ces[w] = S.lbB[row[w]];
                }
            }
        }
        if (mode == 1) dir = choose_dir<NW>(RULE ? RULE : srch.branch_mode, line, best, cbs, ces, valid);
    }

    if (SAMPLE && rec) {
        const int n = T.n;
        int* sch = rec + PBB_SAMPLE_HDR;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (valid[w]) {
                const int u = row[w];
                sch[f + w * 32 + lane] = u;
                sch[n + u] = cbw[w];
                sch[2 * n + u] = cew[w];
                sch[3 * n + u] = cbs[w];
                sch[4 * n + u] = ces[w];
            }
        }
        if (lane == 0) rec[4] = dir;
        __syncwarp();
    }

    // prune: mark children whose bound reaches the incumbent (eliminateJobs :338-410)
#pragma unroll
    for (int w = 0; w < NW; w++) {
        int c1, c2;
        if (mode == 1) { c1 = dir ? ces[w] : cbs[w]; c2 = c1; }
        else if (mode == 0) { c1 = dir ? cew[w] : cbw[w]; c2 = c1; }
        else { c1 = dir ? cew[w] : cbw[w]; c2 = dir ? ces[w] : cbs[w]; }
        bool cut = fa ? (c1 > best || c2 > best) : (c1 >= best || c2 >= best);
        if (valid[w] && cut) row[w] = cell_flag(row[w]);
    }
    if (SORT && srch.sort_nodes) {
        // sortedDFS >= 1: eliminateJobs sorts the row (ivm_bound.cpp:338-370)
        // by the chosen side's first cost, then (2, 4) by the sibling
        // priority chooseChildrenSet set (:506-544), or (3) by the priority
        // alone; out of line to keep the hot loop small.  The first cost is
        // also the cost the side was chosen from (weak, or Johnson in mode 1).
        unsigned long long key[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            const int mine = (mode == 1) ? (dir ? ces[w] : cbs[w]) : (dir ? cew[w] : cbw[w]);
            int prio = 0;
            if (srch.sort_nodes >= 2) {
                const int other = (mode == 1) ? (dir ? cbs[w] : ces[w]) : (dir ? cbw[w] : cew[w]);
                if (srch.sort_crit == 1) prio = mine;
                else if (srch.sort_crit == 2) prio = mine - other;
                else if (mine <= 0) prio = 99999;
                else if (valid[w]) {
                    // the row is flagged already (pruned cells hold -j-1): the
                    // reference sorts before pruning, so take the job itself
                    const int u = cell_job(row[w]);
                    prio = dir ? weak_back_idle(T, S, u) : weak_front_idle(T, S, u);
                }
            }
            const unsigned long long lo = (unsigned)prio ^ 0x80000000u;   // signed order as unsigned
            key[w] = srch.sort_nodes == 3 ? lo : ((unsigned long long)(unsigned)mine << 32) | lo;
        }
        sort_cells(S.rowj, k, key[0], NW > 1 ? key[NW - 1] : 0ull, row[0], NW > 1 ? row[NW - 1] : 0);
#pragma unroll
        for (int w = 0; w < NW; w++)
            if (valid[w]) row[w] = (signed char)S.rowj[w * 32 + lane];
        __syncwarp();
    } else if (prev_dir != dir) {
        // reverse the row when the side changes from the previous level (:620-636)
        int nr[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) {
            int idx = w * 32 + lane;
            int src = k - 1 - idx;
            int v = vgather<NW>(row, src < 0 ? 0 : src);
            nr[w] = (idx < k) ? v : row[w];
        }
#pragma unroll
        for (int w = 0; w < NW; w++) row[w] = nr[w];
    }
    return dir;
}

}  // namespace pbb
