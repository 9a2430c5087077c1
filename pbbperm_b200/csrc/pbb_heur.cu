// Initial upper bounds on the device: NEH (heuristic/src/fastNEH.cpp:230-243
// for the insertion procedure), one warp per instance, for many instances in
// one launch -- the pool computes its admissions' bounds this way, without a
// host round trip, and the engine can start from it.
//
// Insertion of job x into a sequence of `len` jobs uses Taillard's heads and
// tails (fastNEH.cpp:100-178 computeHeads / computeTails / insertJob /
// findBestPos restated): with e the heads of the sequence and q its tails,
// inserting x at position i gives the makespan
//   max_k ( f_k + q_i,k ),  f_k = max(f_{k-1}, e_{i-1,k}) + p_k(x),
// exactly the makespan of the sequence with x at i.  Heads and tails are
// max-plus prefix / suffix scans over the machines (one machine per lane), the
// insertion costs one position per lane.  Integer only: the result equals the
// host restatement pbb_neh job for job.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "pbb_types.h"
#include "pbb_heur.h"
#include "pbb_devguard.h"
#include "pbb_tables.h"
#include "../../include/pbbperm.h"

namespace {

#define HEUR_FULL 0xffffffffu

__device__ __forceinline__ int hlane() { return threadIdx.x & 31; }

// heads after appending a job with times pu (lane = machine, m lanes used):
// h_k = max(h_{k-1}, prev_k) + pu_k, h_{-1} = 0
__device__ __forceinline__ int scan_append(int prev, int pu)
{
    const int lane = hlane();
    int P = pu;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(HEUR_FULL, P, o);
        if (lane >= o) P += t;
    }
    int x = prev - (P - pu);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(HEUR_FULL, x, o);
        if (lane >= o) x = max(x, t);
    }
    return P + max(x, 0);
}

// tails after putting a job first: t_k = max(t_{k+1}, prev_k) + pu_k, t_m = 0
// (lanes >= m carry pu = 0 and prev = 0, so they add nothing)
__device__ __forceinline__ int scan_prepend(int prev, int pu)
{
    const int lane = hlane();
    int Q = pu;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_down_sync(HEUR_FULL, Q, o);
        if (lane + o < 32) Q += t;
    }
    int x = prev - (Q - pu);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_down_sync(HEUR_FULL, x, o);
        if (lane + o < 32) x = max(x, t);
    }
    return Q + max(x, 0);
}

// makespan of seq[0..len) (lane = machine), read by every lane
__device__ __forceinline__ int seq_makespan(const int* p, int n, int m, const int* seq, int len)
{
    const int lane = hlane();
    int h = 0;
    for (int i = 0; i < len; i++) h = scan_append(h, lane < m ? p[lane * n + seq[i]] : 0);
    return __shfl_sync(HEUR_FULL, h, m - 1);
}

}  // namespace

namespace {

// Heads E[i] (positions 0..len-1) and tails Q[i] (0..len, Q[len] = 0) of
// seq[0..len), one machine per lane, stored by position.
__device__ __forceinline__ void heads_tails(const int* p, int n, int m, const int* seq, int len, int* E, int* Q)
{
    const int lane = hlane();
    int h = 0;
    for (int i = 0; i < len; i++) {
        h = scan_append(h, lane < m ? p[lane * n + seq[i]] : 0);
        E[i * 32 + lane] = h;
    }
    int q = 0;
    Q[len * 32 + lane] = 0;
    for (int i = len - 1; i >= 0; i--) {
        q = scan_prepend(q, lane < m ? p[lane * n + seq[i]] : 0);
        Q[i * 32 + lane] = q;
    }
    __syncwarp();
}

// Makespan of x inserted at the best position in [lo, hi] of the sequence
// whose heads and tails are E, Q (fastNEH.cpp:120-178): the first position
// of least makespan.  Returns (makespan << 32) | position, on every lane.
__device__ __forceinline__ unsigned long long best_insert(const int* p, int n, int m, const int* E, const int* Q,
                                                          int x, int lo, int hi)
{
    unsigned long long best = ~0ull;
    for (int i = lo + hlane(); i <= hi; i += 32) {
        int f = 0, c = 0;
        for (int k = 0; k < m; k++) {
            f = max(f, i > 0 ? E[(i - 1) * 32 + k] : 0) + p[k * n + x];
            c = max(c, f + Q[i * 32 + k]);
        }
        const unsigned long long key = ((unsigned long long)(unsigned)c << 32) | (unsigned)i;
        best = key < best ? key : best;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(HEUR_FULL, best, o);
        best = other < best ? other : best;
    }
    return best;
}

// seq[0..len) -> seq[0..len] with x at position pos
__device__ __forceinline__ void insert_at(int* seq, int len, int pos, int x)
{
    const int lane = hlane();
    int moved[2];
    for (int w = 0; w < 2; w++) {
        const int i = w * 32 + lane;
        moved[w] = (i >= pos && i < len) ? seq[i] : -1;
    }
    __syncwarp();
    for (int w = 0; w < 2; w++) {
        const int i = w * 32 + lane;
        if (moved[w] >= 0) seq[i + 1] = moved[w];
    }
    if (lane == 0) seq[pos] = x;
    __syncwarp();
}

// seq[0..len) -> seq[0..len-1) without position pos; returns the job removed
__device__ __forceinline__ int remove_at(int* seq, int len, int pos)
{
    const int lane = hlane();
    const int x = seq[pos];
    int moved[2];
    for (int w = 0; w < 2; w++) {
        const int i = w * 32 + lane;
        moved[w] = (i > pos && i < len) ? seq[i] : -1;
    }
    __syncwarp();
    for (int w = 0; w < 2; w++) {
        const int i = w * 32 + lane;
        if (moved[w] >= 0) seq[i - 1] = moved[w];
    }
    __syncwarp();
    return x;
}

struct HeurSmem {
    int *p, *E, *Q, *seq, *order, *tot, *cur, *best, *vo;
};

__device__ __forceinline__ HeurSmem heur_smem(int* hs)
{
    HeurSmem S;
    S.p = hs;                                   // [m][n]
    S.E = S.p + PBB_MAX_N * PBB_MAX_M;          // [PBB_MAX_N][32] heads by position
    S.Q = S.E + PBB_MAX_N * 32;                 // [PBB_MAX_N + 1][32] tails by position
    S.seq = S.Q + (PBB_MAX_N + 1) * 32;         // [PBB_MAX_N] each of the following
    S.order = S.seq + PBB_MAX_N;
    S.tot = S.order + PBB_MAX_N;
    S.cur = S.tot + PBB_MAX_N;
    S.best = S.cur + PBB_MAX_N;
    S.vo = S.best + PBB_MAX_N;
    return S;
}

// NEH into S.seq; returns the makespan (every lane)
__device__ int neh_warp(const HeurSmem& S, int n, int m)
{
    const int lane = hlane();
    const int* p = S.p;
    // total time per job, then the jobs by decreasing total (ties: lower id first)
    for (int j = lane; j < n; j += 32) {
        int s = 0;
        for (int k = 0; k < m; k++) s += p[k * n + j];
        S.tot[j] = s;
    }
    __syncwarp();
    for (int j = lane; j < n; j += 32) {
        int r = 0;
        for (int i = 0; i < n; i++) r += (S.tot[i] > S.tot[j] || (S.tot[i] == S.tot[j] && i < j)) ? 1 : 0;
        S.order[r] = j;
    }
    __syncwarp();
    int len;
    if (n == 1) {
        if (lane == 0) S.seq[0] = S.order[0];
        __syncwarp();
        len = 1;
    } else {
        // the first two keep the swapped order unless the original one is
        // strictly better (fastNEH.cpp:233-236)
        if (lane == 0) { S.seq[0] = S.order[0]; S.seq[1] = S.order[1]; }
        __syncwarp();
        const int ca = seq_makespan(p, n, m, S.seq, 2);
        if (lane == 0) { S.seq[0] = S.order[1]; S.seq[1] = S.order[0]; }
        __syncwarp();
        const int cb = seq_makespan(p, n, m, S.seq, 2);
        if (ca < cb && lane == 0) { S.seq[0] = S.order[0]; S.seq[1] = S.order[1]; }
        __syncwarp();
        len = 2;
    }
    for (; len < n; len++) {
        const int x = S.order[len];
        heads_tails(p, n, m, S.seq, len, S.E, S.Q);
        const unsigned long long b = best_insert(p, n, m, S.E, S.Q, x, 0, len);
        insert_at(S.seq, len, (int)(b & 0xffffffffu), x);
    }
    return seq_makespan(p, n, m, S.seq, n);
}

// splitmix64 step (the project's generator), lane 0 only
__device__ __forceinline__ unsigned long long rng_next(unsigned long long& s)
{
    s += 0x9E3779B97F4A7C15ull;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// uniform integer in [a, b] from the high word of a 64x(b-a+1) product
__device__ __forceinline__ int rng_range(unsigned long long& s, int a, int b)
{
    return a + (int)__umul64hi(rng_next(s), (unsigned long long)(b - a + 1));
}

}  // namespace

// One warp per task.  Dynamic shared memory: PBB_HEUR_SMEM bytes.
__global__ void __launch_bounds__(32) pbb_neh_kernel(const NehTask* tasks, int count)
{
    extern __shared__ __align__(16) int hs[];
    const int t = blockIdx.x;
    if (t >= count) return;
    const NehTask T = tasks[t];
    const int n = T.n, m = T.m, lane = hlane();
    const HeurSmem S = heur_smem(hs);
    for (int i = lane; i < n * m; i += 32) S.p[i] = T.p[i];
    __syncwarp();
    const int cost = neh_warp(S, n, m);
    for (int i = lane; i < n; i += 32) T.perm[i] = S.seq[i];
    if (lane == 0) {
        if (T.cost) *T.cost = cost;
        if (T.ub) *T.ub = cost;
    }
}

// Iterated greedy from the NEH schedule (heuristic/src/IG.cpp:341-416 runIG,
// destruction :120-160, construction :229-255, localSearchKI :567-612,
// acceptance :258-274), one warp per task.  Every random decision is drawn by
// lane 0 from the task's splitmix64 stream (seed + task index), in this
// order per round: the destruction's window r, its shuffle, then the
// acceptance draw; a worse schedule is kept with probability T / (T + delta),
// T = 0.2 x mean processing time / 10 (the reference's temperature, with the
// exponential replaced by a rational of the same shape so that the test is
// integer arithmetic).  The host restatement in the test oracle follows the
// same stream.
__global__ void __launch_bounds__(32) pbb_ig_kernel(const NehTask* tasks, int count, IgParams prm)
{
    extern __shared__ __align__(16) int hs[];
    const int t = blockIdx.x;
    if (t >= count) return;
    const NehTask T = tasks[t];
    const int n = T.n, m = T.m, lane = hlane();
    const HeurSmem S = heur_smem(hs);
    __shared__ int removed[PBB_MAX_N];
    for (int i = lane; i < n * m; i += 32) S.p[i] = T.p[i];
    __syncwarp();
    int cur_cost = neh_warp(S, n, m);
    int best_cost = cur_cost;
    long long sum = 0;
    for (int i = 0; i < n * m; i++) sum += S.p[i];
    const long long temp1000 = 20 * sum / ((long long)n * m);   // 1000 x 0.2 x mean / 10
    for (int i = lane; i < n; i += 32) { S.cur[i] = S.seq[i]; S.best[i] = S.seq[i]; }
    // visit order: the middle position first, then alternately right and left (IG.cpp:33-45)
    if (lane == 0) {
        const int start = n / 2;
        int ind = 0;
        for (int i = start; i < n; i++) { S.vo[ind] = i; ind += 2; }
        ind = 1;
        for (int i = start - 1; i >= 0; i--) { S.vo[ind] = i; ind += 2; }
    }
    __syncwarp();
    int kmax = 1;
    while ((kmax + 1) * (kmax + 1) <= n) kmax++;   // integer square root
    unsigned long long rs = prm.seed + (unsigned long long)t;
    int perturb = prm.destruct;
    for (int it = 0; it < prm.iterations && n >= 3; it++) {
        const int d = min(perturb, n - 1);
        for (int i = lane; i < n; i += 32) S.seq[i] = S.cur[i];
        __syncwarp();
        // destruction: d positions from a shuffled prefix of the visit order
        if (lane == 0) {
            const int r = rng_range(rs, d, n);
            for (int i = 0; i < r; i++) S.order[i] = S.vo[i];
            for (int i = 0; i < r - 1; i++) {
                const int j = rng_range(rs, i, r - 1);
                const int tmp = S.order[i]; S.order[i] = S.order[j]; S.order[j] = tmp;
            }
            // remove the chosen positions, highest first, keeping their jobs in draw order
            for (int i = 0; i < d; i++) removed[i] = S.seq[S.order[i]];
            for (int i = 0; i < n; i++) S.tot[i] = 0;
            for (int i = 0; i < d; i++) S.tot[S.order[i]] = 1;
            int w = 0;
            for (int i = 0; i < n; i++)
                if (!S.tot[i]) S.seq[w++] = S.seq[i];
        }
        __syncwarp();
        // construction: each removed job at its best position
        int len = n - d;
        for (int i = 0; i < d; i++) {
            const int x = removed[i];
            heads_tails(S.p, n, m, S.seq, len, S.E, S.Q);
            const unsigned long long b = best_insert(S.p, n, m, S.E, S.Q, x, 0, len);
            insert_at(S.seq, len, (int)(b & 0xffffffffu), x);
            len++;
        }
        // local search: move the job at each visited position to the best
        // place within kmax of it, first improvement, until a pass finds none
        int cost = seq_makespan(S.p, n, m, S.seq, n);
        for (int pass = 0; pass < prm.ls_passes; pass++) {
            bool improved = false;
            for (int j = 0; j < n && !improved; j++) {
                const int i = S.vo[j];
                const int x = remove_at(S.seq, n, i);
                heads_tails(S.p, n, m, S.seq, n - 1, S.E, S.Q);
                const unsigned long long b =
                    best_insert(S.p, n, m, S.E, S.Q, x, max(0, i - kmax), min(n - 1, i + kmax));
                const int c = (int)(b >> 32);
                if (c < cost) {
                    insert_at(S.seq, n - 1, (int)(b & 0xffffffffu), x);
                    cost = c;
                    improved = true;
                } else {
                    insert_at(S.seq, n - 1, i, x);
                }
            }
            if (!improved) break;
        }
        // acceptance: one draw per round; not worse, or u / 2^32 < T / (T + delta)
        int accept = 0;
        if (lane == 0) {
            const long long delta = (long long)cost - cur_cost;
            const unsigned long long u = rng_next(rs) >> 32;
            accept = (delta <= 0 ||
                      u < ((unsigned long long)temp1000 << 32) / (unsigned long long)(temp1000 + 1000 * delta)) ? 1 : 0;
        }
        accept = __shfl_sync(HEUR_FULL, accept, 0);
        if (accept) {
            for (int i = lane; i < n; i += 32) S.cur[i] = S.seq[i];
            cur_cost = cost;
            perturb = prm.destruct;
        } else {
            perturb = perturb + 1 > prm.destruct_max ? prm.destruct : perturb + 1;
        }
        if (cost < best_cost) {
            best_cost = cost;
            for (int i = lane; i < n; i += 32) S.best[i] = S.seq[i];
        }
        __syncwarp();
    }
    for (int i = lane; i < n; i += 32) T.perm[i] = S.best[i];
    if (lane == 0) {
        if (T.cost) *T.cost = best_cost;
        if (T.ub) *T.ub = best_cost;
    }
}

namespace pbbl {

cudaError_t launch_neh(const NehTask* tasks_d, int count, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    cudaFuncSetAttribute(pbb_neh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PBB_HEUR_SMEM);
    pbb_neh_kernel<<<count, 32, PBB_HEUR_SMEM, st>>>(tasks_d, count);
    return cudaGetLastError();
}

cudaError_t launch_ig(const NehTask* tasks_d, int count, const IgParams& prm, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    cudaFuncSetAttribute(pbb_ig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, PBB_HEUR_SMEM);
    pbb_ig_kernel<<<count, 32, PBB_HEUR_SMEM, st>>>(tasks_d, count, prm);
    return cudaGetLastError();
}

}  // namespace pbbl

namespace {

// Heuristic of `count` host instances on `device`; ig NULL = NEH alone.
int heur_batch(const pbb_instance* inst, int32_t count, int32_t device, const IgParams* ig, int32_t* perms,
               int32_t* costs)
{
    if (count < 0 || (count > 0 && (!inst || !perms || !costs))) return pbbt::fail(PBB_E_INVAL, "bad arguments");
    if (count == 0) return PBB_OK;
    size_t words = 0;
    for (int i = 0; i < count; i++) {
        const int n = inst[i].n_jobs, m = inst[i].n_machines;
        if (!inst[i].p || n < 1 || n > PBB_MAX_JOBS || m < 1 || m > PBB_MAX_MACHINES)
            return pbbt::fail(PBB_E_INVAL, "instance size out of range (1..64 jobs, 1..32 machines)");
        const int rc = pbbt::check_times(inst[i].p, n, m);
        if (rc) return rc;
        words += (size_t)n * m;
    }
    pbbh::DeviceGuard keep_callers_device;
    if (cudaSetDevice(device) != cudaSuccess) return pbbt::fail(PBB_E_CUDA, "cudaSetDevice failed");
    cudaStream_t st = nullptr;
    int* buf = nullptr;
    NehTask* tasks_d = nullptr;
    int rc = PBB_OK;
    do {
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            rc = pbbt::fail(PBB_E_CUDA, "stream creation failed");
            break;
        }
        const size_t out_words = (size_t)count * (PBB_MAX_JOBS + 1);
        if (cudaMalloc(&buf, sizeof(int) * (words + out_words)) != cudaSuccess ||
            cudaMalloc(&tasks_d, sizeof(NehTask) * count) != cudaSuccess) {
            rc = pbbt::fail(PBB_E_NOMEM, "device allocation failed");
            break;
        }
        std::vector<int> host(words);
        std::vector<NehTask> tasks(count);
        size_t off = 0;
        int* out = buf + words;
        for (int i = 0; i < count; i++) {
            const int n = inst[i].n_jobs, m = inst[i].n_machines;
            memcpy(host.data() + off, inst[i].p, sizeof(int) * n * m);
            tasks[i].p = buf + off;
            tasks[i].n = n;
            tasks[i].m = m;
            tasks[i].perm = out + (size_t)i * (PBB_MAX_JOBS + 1);
            tasks[i].cost = out + (size_t)i * (PBB_MAX_JOBS + 1) + PBB_MAX_JOBS;
            tasks[i].ub = nullptr;
            off += (size_t)n * m;
        }
        cudaError_t ce = cudaMemcpyAsync(buf, host.data(), sizeof(int) * words, cudaMemcpyHostToDevice, st);
        if (!ce) ce = cudaMemcpyAsync(tasks_d, tasks.data(), sizeof(NehTask) * count, cudaMemcpyHostToDevice, st);
        if (!ce) ce = ig ? pbbl::launch_ig(tasks_d, count, *ig, st) : pbbl::launch_neh(tasks_d, count, st);
        std::vector<int> res(out_words);
        if (!ce) ce = cudaMemcpyAsync(res.data(), out, sizeof(int) * out_words, cudaMemcpyDeviceToHost, st);
        if (!ce) ce = cudaStreamSynchronize(st);
        if (ce) {
            rc = pbbt::fail(PBB_E_CUDA, cudaGetErrorString(ce));
            break;
        }
        for (int i = 0; i < count; i++) {
            for (int j = 0; j < PBB_MAX_JOBS; j++)
                perms[(size_t)i * PBB_MAX_JOBS + j] = j < inst[i].n_jobs ? res[(size_t)i * (PBB_MAX_JOBS + 1) + j] : 0;
            costs[i] = res[(size_t)i * (PBB_MAX_JOBS + 1) + PBB_MAX_JOBS];
        }
    } while (0);
    cudaFree(buf);
    cudaFree(tasks_d);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // namespace

extern "C" int pbb_neh_batch(const pbb_instance* inst, int32_t count, int32_t device, int32_t* perms,
                             int32_t* costs)
{
    return heur_batch(inst, count, device, nullptr, perms, costs);
}

extern "C" int pbb_ig_batch(const pbb_instance* inst, int32_t count, int32_t device, int32_t iterations,
                            uint64_t seed, int32_t* perms, int32_t* costs)
{
    if (iterations < 0 || iterations > 100000) return pbbt::fail(PBB_E_INVAL, "iterations must be in [0, 100000]");
    IgParams prm;
    prm.iterations = iterations;
    prm.destruct = 2;          // IG::destructStrength (heuristic/src/IG.cpp:22)
    prm.destruct_max = 5;      // perturbation cap (IG.cpp:393-396)
    prm.ls_passes = 64;
    prm.seed = seed;
    return heur_batch(inst, count, device, &prm, perms, costs);
}
