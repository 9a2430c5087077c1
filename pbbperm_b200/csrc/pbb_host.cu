// Host side of the engine: instance tables, device memory, launches, and the
// C ABI declared in include/pbbperm.h.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <string>
#include <thread>
#include <vector>

#include "pbb_types.h"
#include "pbb_devguard.h"
#include "pbb_launch.h"
#include "pbb_tables.h"
#include "pbb_heur.h"
#include "../../include/pbbperm.h"
#include "../../include/pbbperm_diag.h"

using pbbt::HostTables;
using pbbt::build_tables;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? PBB_E_NOMEM : PBB_E_CUDA;
}

#define CK(call)                                        \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

struct DeviceInstance {
    int* p = nullptr;
    unsigned long long* je = nullptr;
    unsigned char* pm = nullptr;
    unsigned char* posj = nullptr;
    int* mt = nullptr;
    DevInstance view{};

    int upload(const HostTables& H, cudaStream_t st)
    {
        CK(cudaMalloc(&p, sizeof(int) * H.n * H.m));
        CK(cudaMalloc(&je, sizeof(unsigned long long) * H.je.size()));
        CK(cudaMalloc(&pm, 2 * H.Ppad));
        CK(cudaMalloc(&posj, H.posj.size()));
        CK(cudaMalloc(&mt, sizeof(int) * 2 * H.m));
        CK(cudaMemcpyAsync(p, H.p.data(), sizeof(int) * H.n * H.m, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(je, H.je.data(), sizeof(unsigned long long) * H.je.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(pm, H.pm0.data(), H.Ppad, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(posj, H.posj.data(), H.posj.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(pm + H.Ppad, H.pm1.data(), H.Ppad, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(mt, H.min_arr.data(), sizeof(int) * H.m, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(mt + H.m, H.min_dep.data(), sizeof(int) * H.m, cudaMemcpyHostToDevice, st));
        view.n = H.n; view.m = H.m; view.P = H.P; view.Ppad = H.Ppad;
        view.p = p; view.je = je; view.pm0 = pm; view.pm1 = pm + H.Ppad;
        view.min_arr = mt; view.min_dep = mt + H.m;
        view.posj = posj;
        return PBB_OK;
    }
    void release()
    {
        cudaFree(p); cudaFree(je); cudaFree(pm); cudaFree(mt); cudaFree(posj);
        p = nullptr; je = nullptr; pm = nullptr; mt = nullptr; posj = nullptr;
    }
};

int max_smem_optin(int dev)
{
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

// The most warps per CTA (up to `requested`) whose tables and scratch fit;
// `explorer`: add the per-warp free-position masks when they fit too (the
// explorer runs one CTA per SM, so they never cost a warp).
int pick_warps(const HostTables& H, int requested, int dev, int& smem, bool explorer = false)
{
    const int cap = max_smem_optin(dev);
    int w = requested > 0 ? std::min(requested, PBB_WARPS_MAX) : PBB_WARPS_MAX;
    for (; w >= 1; w--) {
        smem = pbbl::smem_bytes(H.n, H.m, H.Ppad, w);
        if (smem <= cap) {
            const int with_masks = pbbl::smem_bytes(H.n, H.m, H.Ppad, w, 1);
            if (explorer && with_masks <= cap) smem = with_masks;
            return w;
        }
    }
    return 0;
}

}  // namespace

namespace pbbh {
// error message for entry points compiled in other files of the library
void set_error(const char* msg) { g_err = msg; }
}  // namespace pbbh

struct pbb_engine;
namespace pbbh {
// engine facts for the checkpoint code (pbb_ckpt.cu)
int engine_jobs(const pbb_engine* e);
int engine_explorers(const pbb_engine* e);
const std::vector<int32_t>& engine_root(const pbb_engine* e);
void engine_set_start_perm(pbb_engine* e, const int32_t* perm);
}  // namespace pbbh

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
struct pbb_engine {
    pbb_config cfg{};
    HostTables H;
    int dev = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int nw = 2, warps = 0, ctas = 0, smem = 0, root_smem = 0;
    DeviceInstance di;
    signed char *mat = nullptr, *vec = nullptr, *bestperm = nullptr;
    int* path = nullptr;   // per explorer and level: heads, tails, free loads
    int *line = nullptr, *state = nullptr, *bestcost = nullptr, *qval = nullptr, *ub_d = nullptr, *root_d = nullptr;
    int* ival_d = nullptr;   // [2][64] interval start / end vectors
    unsigned* qseq = nullptr;
    GroupCtl* ctl = nullptr;
    DevGroup* group_d = nullptr;
    int* ngroups_d = nullptr;     // device copy of the group count (1)
    DevGroup group{};
    double dev_seconds = 0.0;
    bool started = false, done = false;
    int32_t ub = INT32_MAX;
    double slice_s = 2.0;
    int select_budget = 4096;
    int max_rounds = INT_MAX;      // explorer loop rounds per launch
    int* neh_d = nullptr;          // device NEH result: perm[64], cost
    NehTask* neh_task_d = nullptr; // the engine's instance as a heuristic task
    bool from_neh = false;         // the current search started from PBB_UB_NEH
    std::vector<int32_t> root;     // root permutation of the current search
    std::vector<int32_t> start_perm;   // schedule of the starting bound (e.g. a checkpoint's incumbent)
    SampleBuf* sample_d = nullptr; // node sampling (diagnostic), NULL when off
    int* sample_rec = nullptr;
    int sample_stride = 0;
    double wait_limit_s = -1.0;    // host wait per window: < 0 window + 60 s, 0 unbounded
    bool pending = false;          // a window whose wait ran out is still on the stream
};

namespace pbbh {
int engine_jobs(const pbb_engine* e) { return e->H.n; }
int engine_explorers(const pbb_engine* e) { return e->cfg.nb_ivms; }
const std::vector<int32_t>& engine_root(const pbb_engine* e) { return e->root; }
void engine_set_start_perm(pbb_engine* e, const int32_t* perm) { e->start_perm.assign(perm, perm + e->H.n); }
}  // namespace pbbh

namespace {

// Wait for `ev` with a host-side deadline: PBB_E_TIMEOUT when it has not
// completed after limit_s seconds (limit_s <= 0: wait without limit).  Polls
// with a short sleep so that the waiting thread does not spin a core.
int wait_event(cudaEvent_t ev, double limit_s)
{
    if (limit_s <= 0) {
        CK(cudaEventSynchronize(ev));
        return PBB_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    unsigned sleep_us = 20;
    while (true) {
        const cudaError_t q = cudaEventQuery(ev);
        if (q == cudaSuccess) return PBB_OK;
        if (q != cudaErrorNotReady) return cuda_fail(q, "exploration window");
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > limit_s) return PBB_E_TIMEOUT;
        std::this_thread::sleep_for(std::chrono::microseconds(sleep_us));
        sleep_us = std::min(2 * sleep_us, 500u);
    }
}

// Account a window whose host wait ran out: it ends by its own device-time
// budget, so this blocks for at most the rest of that budget.
int settle(pbb_engine* e)
{
    if (!e->pending) return PBB_OK;
    CK(cudaEventSynchronize(e->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
    e->dev_seconds += ms * 1e-3;
    int active = 0;
    CK(cudaMemcpy(&active, &e->ctl->active, sizeof(int), cudaMemcpyDeviceToHost));
    e->done = (active == 0);
    e->pending = false;
    return PBB_OK;
}

}  // namespace

extern "C" {

void pbb_config_default(pbb_config* c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->bounding_mode = 2;
    c->branching_mode = 3;
    c->find_all = 0;
    c->johnson_mode = 0;
    c->early_stop_johnson = 0;
    c->sorted_dfs = 0;
    c->sorting_criterion = 1;
    c->nb_ivms = 16384;
    c->device = 0;
}

const char* pbb_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace pbbh {
// Search settings every entry point accepts (engine and pool).
// earlyStopJohnson: a child's Johnson scan stops once its running maximum
// exceeds the incumbent (bound_fsp_strong.cpp:154-158); that child is pruned
// either way, so node counts do not change -- except with the Johnson bound
// choosing the side by MaxSum (boundingMode 1, adaptiveBranchingMode 1),
// where the pruned children's partial values enter the choice and, in the
// reference, depend on each thread's machine-pair success history
// (:112-122): that combination is rejected.
int check_search(const pbb_config* c)
{
    if (c->bounding_mode < 0 || c->bounding_mode > 2) return fail(PBB_E_INVAL, "boundingMode must be 0, 1 or 2");
    const int b = c->branching_mode;
    if (!(b == -3 || b == -2 || b == -1 || b == 1 || b == 2 || b == 3))
        return fail(PBB_E_INVAL, "adaptiveBranchingMode must be one of -3,-2,-1,1,2,3");
    if (c->early_stop_johnson && c->bounding_mode == 1 && b == 1)
        return fail(PBB_E_UNSUPPORTED, "earlyStopJohnson=true with boundingMode=1 and MaxSum branching is not "
                                       "supported (the side choice would depend on a thread's pair-order history)");
    if (c->sorted_dfs < 0 || c->sorted_dfs > 4) return fail(PBB_E_INVAL, "sortedDFS must be in 0..4");
    if (c->sorted_dfs >= 2) {
        // the sibling priorities of chooseChildrenSet (ivm_bound.cpp:506-544)
        const int k = c->sorting_criterion;
        if (k == 4)
            return fail(PBB_E_UNSUPPORTED, "sortingCriterion=4 is not supported: the reference's completeSchedule "
                                           "writes past the node's free jobs, so its priorities are not defined");
        if (k < 1 || k > 4) return fail(PBB_E_INVAL, "sortingCriterion must be 1, 2 or 3 with sortedDFS >= 2");
        if (k == 3 && c->bounding_mode == 1)
            return fail(PBB_E_UNSUPPORTED, "sortingCriterion=3 with boundingMode=1 is not supported: the reference "
                                           "reads an unset Johnson idle time for children with one free job");
        if (k == 2 && c->bounding_mode == 1 && c->early_stop_johnson)
            return fail(PBB_E_UNSUPPORTED, "sortingCriterion=2 with boundingMode=1 and earlyStopJohnson=true is not "
                                           "supported: the priority would read a pruned side's partial bound");
    }
    return PBB_OK;
}
}  // namespace pbbh

extern "C" {

static int check_config(const pbb_config* c)
{
    const int rc = pbbh::check_search(c);
    if (rc) return rc;
    if (c->nb_ivms < 1 || c->nb_ivms > (1 << 22)) return fail(PBB_E_INVAL, "nbIVMs must be in [1, 4194304]");
    return PBB_OK;
}

int pbb_engine_destroy(pbb_engine* e)
{
    if (!e) return PBB_OK;
    pbbh::DeviceGuard keep_callers_device;
    cudaSetDevice(e->dev);
    if (e->st) cudaStreamSynchronize(e->st);
    e->di.release();
    cudaFree(e->mat); cudaFree(e->vec); cudaFree(e->bestperm); cudaFree(e->path);
    cudaFree(e->line); cudaFree(e->state); cudaFree(e->bestcost); cudaFree(e->qval); cudaFree(e->qseq);
    cudaFree(e->ub_d); cudaFree(e->root_d); cudaFree(e->ival_d); cudaFree(e->ctl); cudaFree(e->group_d);
    cudaFree(e->ngroups_d);
    cudaFree(e->sample_d);
    cudaFree(e->sample_rec);
    cudaFree(e->neh_d);
    cudaFree(e->neh_task_d);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->st) cudaStreamDestroy(e->st);
    delete e;
    return PBB_OK;
}

static int engine_create(const pbb_instance* inst, const pbb_config* cfg, pbb_engine* e)
{
    e->cfg = *cfg;
    int rc = check_config(cfg);
    if (rc) return rc;
    rc = build_tables(inst, cfg->johnson_mode, e->H);
    if (rc) return rc;
    e->dev = cfg->device;
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    CK(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&e->ev0));
    CK(cudaEventCreate(&e->ev1));
    const HostTables& H = e->H;
    e->nw = H.n <= 32 ? 1 : 2;
    e->warps = pick_warps(H, cfg->warps_per_cta, e->dev, e->smem, true);
    if (e->warps < 1) return fail(PBB_E_INVAL, "instance tables do not fit in shared memory");
    e->root_smem = pbbl::smem_bytes(H.n, H.m, H.Ppad, 1);
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->dev));
    e->ctas = cfg->ctas > 0 ? cfg->ctas : sms;
    rc = e->di.upload(H, e->st);
    if (rc) return rc;
    const int B = cfg->nb_ivms;
    const int npad = PBB_MAX_N;
    CK(cudaMalloc(&e->mat, (size_t)B * npad * npad));
    CK(cudaMalloc(&e->vec, (size_t)B * npad * 4));
    CK(cudaMalloc(&e->path, (size_t)B * npad * PBB_PATH_INTS * sizeof(int)));
    CK(cudaMalloc(&e->bestperm, (size_t)B * npad));
    CK(cudaMalloc(&e->line, sizeof(int) * B));
    CK(cudaMalloc(&e->state, sizeof(int) * B));
    CK(cudaMalloc(&e->bestcost, sizeof(int) * B));
    CK(cudaMalloc(&e->qval, sizeof(int) * B));
    CK(cudaMalloc(&e->qseq, sizeof(unsigned) * B));
    CK(cudaMalloc(&e->ub_d, sizeof(int)));
    CK(cudaMalloc(&e->root_d, sizeof(int) * PBB_MAX_N));
    CK(cudaMalloc(&e->neh_d, sizeof(int) * (PBB_MAX_N + 1)));
    CK(cudaMalloc(&e->neh_task_d, sizeof(NehTask)));
    {
        NehTask t;
        t.p = e->di.p;
        t.n = H.n;
        t.m = H.m;
        t.perm = e->neh_d;
        t.cost = e->neh_d + PBB_MAX_N;
        t.ub = e->ub_d;
        CK(cudaMemcpyAsync(e->neh_task_d, &t, sizeof(t), cudaMemcpyHostToDevice, e->st));
    }
    CK(cudaMalloc(&e->ival_d, sizeof(int) * 2 * PBB_MAX_N));
    CK(cudaMalloc(&e->ctl, sizeof(GroupCtl)));
    CK(cudaMalloc(&e->group_d, sizeof(DevGroup)));
    CK(cudaMalloc(&e->ngroups_d, sizeof(int)));
    {
        const int one = 1;
        CK(cudaMemcpyAsync(e->ngroups_d, &one, sizeof(int), cudaMemcpyHostToDevice, e->st));
    }
    CK(cudaMemsetAsync(e->mat, 0, (size_t)B * npad * npad, e->st));
    DevGroup& g = e->group;
    g.inst = e->di.view;
    g.search.bound_mode = cfg->bounding_mode;
    g.search.branch_mode = cfg->branching_mode;
    g.search.find_all = cfg->find_all ? 1 : 0;
    g.search.sort_nodes = cfg->sorted_dfs;
    g.search.sort_crit = cfg->sorting_criterion;
    g.search.core_warps = cfg->core_warps > 0 ? cfg->core_warps : PBB_CORE_WARPS;
    g.search.split_depth = cfg->split_depth > 0 ? cfg->split_depth : PBB_SPLIT_DEPTH;
    g.search.share_after = cfg->share_after > 0 ? cfg->share_after : (cfg->share_after < 0 ? 0 : PBB_SHARE_AFTER);
    g.search.early_stop = cfg->early_stop_johnson ? 1 : 0;
    g.ivm.count = B;
    g.ivm.npad = npad;
    g.ivm.mat = e->mat;
    g.ivm.pos = e->vec;
    g.ivm.end = e->vec + (size_t)B * npad;
    g.ivm.dir = e->vec + (size_t)2 * B * npad;
    g.ivm.pj = e->vec + (size_t)3 * B * npad;
    g.ivm.line = e->line;
    g.ivm.state = e->state;
    g.ivm.bestcost = e->bestcost;
    g.ivm.bestperm = e->bestperm;
    g.ivm.qseq = e->qseq;
    g.ivm.qval = e->qval;
    g.ivm.path = e->path;
    g.ctl = e->ctl;
    g.first_cta = 0;
    g.ctas = e->ctas;
    CK(cudaMemcpyAsync(e->group_d, &g, sizeof(DevGroup), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    return PBB_OK;
}

int pbb_engine_create(const pbb_instance* inst, const pbb_config* cfg, pbb_engine** out)
{
    if (!out) return fail(PBB_E_INVAL, "out is NULL");
    *out = nullptr;
    pbb_config def;
    if (!cfg) { pbb_config_default(&def); cfg = &def; }
    pbb_engine* e = new pbb_engine();
    int rc = engine_create(inst, cfg, e);
    if (rc) {
        std::string keep = g_err;
        pbb_engine_destroy(e);
        g_err = keep;
        return rc;
    }
    *out = e;
    return PBB_OK;
}

static int start_impl(pbb_engine* e, int32_t ub, const int32_t* root_perm, const int32_t* pos, const int32_t* end)
{
    if (!e) return fail(PBB_E_INVAL, "engine is NULL");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    const int n = e->H.n;
    std::vector<int> root(PBB_MAX_N, 0);
    std::vector<int> seen(n, 0);
    for (int i = 0; i < n; i++) {
        const int j = root_perm ? root_perm[i] : i;
        if (j < 0 || j >= n || seen[j]) return fail(PBB_E_INVAL, "root_perm is not a permutation of 0..n-1");
        seen[j] = 1;
        root[i] = j;
    }
    // factoradic interval: digit i in [0, n-i) (sequentialbb.cpp:207-222 checks)
    std::vector<int> iv(2 * PBB_MAX_N, 0);
    for (int i = 0; i < n; i++) {
        const int p = pos ? pos[i] : 0;
        const int q = end ? end[i] : n - 1 - i;
        if (p < 0 || p >= n - i || q < 0 || q >= n - i) return fail(PBB_E_INVAL, "interval digit out of range");
        iv[i] = p;
        iv[PBB_MAX_N + i] = q;
    }
    if (ub < 0 && ub != PBB_UB_NEH) return fail(PBB_E_INVAL, "ub must be >= 0 (or PBB_UB_NEH)");
    e->ub = ub;
    e->from_neh = ub == PBB_UB_NEH;
    e->root.assign(root.begin(), root.begin() + n);
    e->start_perm.clear();
    CK(cudaMemcpyAsync(e->ub_d, &ub, sizeof(int), cudaMemcpyHostToDevice, e->st));
    // the device NEH writes its makespan where the reset kernel reads the bound
    if (e->from_neh) CK(pbbl::launch_neh(e->neh_task_d, 1, e->st));
    CK(cudaMemcpyAsync(e->root_d, root.data(), sizeof(int) * PBB_MAX_N, cudaMemcpyHostToDevice, e->st));
    CK(cudaMemcpyAsync(e->ival_d, iv.data(), sizeof(int) * 2 * PBB_MAX_N, cudaMemcpyHostToDevice, e->st));
    CK(pbbl::launch_reset(e->group_d, 1, e->ub_d, e->st));
    CK(pbbl::launch_root(e->nw, e->group_d, 1, e->root_d, e->ival_d, PBB_MAX_N, e->root_smem, e->st));
    CK(cudaStreamSynchronize(e->st));
    if (e->from_neh) CK(cudaMemcpy(&e->ub, e->ub_d, sizeof(int), cudaMemcpyDeviceToHost));
    e->pending = false;
    GroupCtl c;
    CK(cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    e->started = true;
    e->done = (c.active == 0);
    e->dev_seconds = 0.0;
    return PBB_OK;
}

int pbb_start(pbb_engine* e, int32_t ub, const int32_t* root_perm) { return start_impl(e, ub, root_perm, nullptr, nullptr); }

int pbb_start_interval(pbb_engine* e, int32_t ub, const int32_t* root_perm, const int32_t* pos, const int32_t* end)
{
    if (!pos || !end) return fail(PBB_E_INVAL, "pos/end are NULL");
    return start_impl(e, ub, root_perm, pos, end);
}

int pbb_init_from_fac(pbb_engine* e, int32_t ub, const int32_t* root_perm, int32_t nb_intervals, const int32_t* ids,
                      const int32_t* pos, const int32_t* end)
{
    if (!e) return fail(PBB_E_INVAL, "engine is NULL");
    if (!pos || !end) return fail(PBB_E_INVAL, "pos/end are NULL");
    const int B = e->cfg.nb_ivms;
    if (nb_intervals < 1 || nb_intervals > B) return fail(PBB_E_INVAL, "nb_intervals must be in [1, nb_ivms]");
    if (ub < 0 && ub != PBB_UB_NEH) return fail(PBB_E_INVAL, "ub must be >= 0 (or PBB_UB_NEH)");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    const int n = e->H.n;
    std::vector<int> root(PBB_MAX_N, 0);
    std::vector<int> seen(n, 0);
    for (int i = 0; i < n; i++) {
        const int j = root_perm ? root_perm[i] : i;
        if (j < 0 || j >= n || seen[j]) return fail(PBB_E_INVAL, "root_perm is not a permutation of 0..n-1");
        seen[j] = 1;
        root[i] = j;
    }
    std::vector<int> iv((size_t)2 * nb_intervals * PBB_MAX_N, 0);
    std::vector<int> id(nb_intervals);
    std::vector<char> taken(B, 0);
    for (int k = 0; k < nb_intervals; k++) {
        const int x = ids ? ids[k] : k;
        if (x < 0 || x >= B || taken[x]) return fail(PBB_E_INVAL, "ids must be distinct explorers < nb_ivms");
        taken[x] = 1;
        id[k] = x;
        for (int i = 0; i < n; i++) {
            const int p = pos[(size_t)k * n + i], q = end[(size_t)k * n + i];
            if (p < 0 || p >= n - i || q < 0 || q >= n - i) return fail(PBB_E_INVAL, "interval digit out of range");
            iv[(size_t)(2 * k) * PBB_MAX_N + i] = p;
            iv[(size_t)(2 * k + 1) * PBB_MAX_N + i] = q;
        }
    }
    int* ival_d = nullptr;
    int* ids_d = nullptr;
    CK(cudaMalloc(&ival_d, sizeof(int) * iv.size()));
    cudaError_t err = cudaMalloc(&ids_d, sizeof(int) * nb_intervals);
    if (!err) err = cudaMemcpyAsync(ival_d, iv.data(), sizeof(int) * iv.size(), cudaMemcpyHostToDevice, e->st);
    if (!err) err = cudaMemcpyAsync(ids_d, id.data(), sizeof(int) * nb_intervals, cudaMemcpyHostToDevice, e->st);
    if (!err) err = cudaMemcpyAsync(e->ub_d, &ub, sizeof(int), cudaMemcpyHostToDevice, e->st);
    if (!err && ub == PBB_UB_NEH) err = pbbl::launch_neh(e->neh_task_d, 1, e->st);
    if (!err) err = cudaMemcpyAsync(e->root_d, root.data(), sizeof(int) * PBB_MAX_N, cudaMemcpyHostToDevice, e->st);
    if (!err) err = pbbl::launch_reset(e->group_d, 1, e->ub_d, e->st);
    if (!err)
        err = pbbl::launch_root(e->nw, e->group_d, 1, e->root_d, ival_d, PBB_MAX_N, e->root_smem, e->st,
                                nb_intervals, ids_d);
    if (!err) err = cudaStreamSynchronize(e->st);
    if (!err) e->pending = false;
    cudaFree(ival_d);
    cudaFree(ids_d);
    if (err) return fail(PBB_E_CUDA, std::string("init_from_fac: ") + cudaGetErrorString(err));
    GroupCtl c;
    CK(cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    e->ub = ub;
    e->from_neh = ub == PBB_UB_NEH;
    if (e->from_neh) CK(cudaMemcpy(&e->ub, e->ub_d, sizeof(int), cudaMemcpyDeviceToHost));
    e->root.assign(root.begin(), root.begin() + n);
    e->start_perm.clear();
    e->started = true;
    e->done = (c.active == 0);
    e->dev_seconds = 0.0;
    return PBB_OK;
}

int pbb_get_intervals(pbb_engine* e, int32_t max_intervals, int32_t* pos, int32_t* end, int32_t* ids,
                      int32_t* nb_intervals)
{
    if (!e || !e->started) return fail(PBB_E_INVAL, "engine not started");
    if (!nb_intervals) return fail(PBB_E_INVAL, "nb_intervals is NULL");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(cudaStreamSynchronize(e->st));
    const int B = e->cfg.nb_ivms, n = e->H.n;
    std::vector<int> st(B);
    std::vector<signed char> ps((size_t)B * PBB_MAX_N), es((size_t)B * PBB_MAX_N);
    CK(cudaMemcpy(st.data(), e->state, sizeof(int) * B, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ps.data(), e->group.ivm.pos, ps.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(es.data(), e->group.ivm.end, es.size(), cudaMemcpyDeviceToHost));
    // An explorer stopped between selection steps may hold a digit one past
    // its level's last cell (n - l: "this level is done"); carry it into the
    // level above (ivm::goUp, multicore/src/ivm.cpp:56-72) so that every
    // exported digit lies in [0, n - l), and drop intervals the carry empties.
    std::vector<int> keep;
    std::vector<int> pv((size_t)B * n), ev((size_t)B * n);
    for (int k = 0; k < B; k++) {
        if (st[k] != IVM_ACTIVE) continue;
        int* a = &pv[(size_t)k * n];
        int* z = &ev[(size_t)k * n];
        for (int i = 0; i < n; i++) {
            a[i] = ps[(size_t)k * PBB_MAX_N + i];
            z[i] = es[(size_t)k * PBB_MAX_N + i];
        }
        for (int l = n - 1; l > 0; l--)
            if (a[l] >= n - l) { a[l] = 0; a[l - 1]++; }
        if (a[0] >= n) continue;
        bool le = true;     // pos <= end, lexicographically
        for (int l = 0; l < n; l++)
            if (a[l] != z[l]) { le = a[l] < z[l]; break; }
        if (le) keep.push_back(k);
    }
    const int cnt = (int)keep.size();
    *nb_intervals = cnt;
    if (cnt > max_intervals) return fail(PBB_E_INVAL, "buffer too small for the active intervals");
    if (cnt > 0 && (!pos || !end)) return fail(PBB_E_INVAL, "pos/end are NULL");
    for (int w = 0; w < cnt; w++) {
        const int k = keep[w];
        for (int i = 0; i < n; i++) {
            pos[(size_t)w * n + i] = pv[(size_t)k * n + i];
            end[(size_t)w * n + i] = ev[(size_t)k * n + i];
        }
        if (ids) ids[w] = k;
    }
    return PBB_OK;
}

int pbb_set_ub(pbb_engine* e, int32_t ub)
{
    if (!e || !e->started) return fail(PBB_E_INVAL, "engine not started");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(pbbl::launch_lower_ub(e->group_d, 0, ub, e->st));
    CK(cudaStreamSynchronize(e->st));
    return PBB_OK;
}

int pbb_set_wait_limit(pbb_engine* e, double seconds)
{
    if (!e) return fail(PBB_E_INVAL, "engine is NULL");
    e->wait_limit_s = seconds;
    return PBB_OK;
}

int pbb_diag_set_step_limits(pbb_engine* e, int32_t select_budget, int32_t max_rounds)
{
    if (!e) return fail(PBB_E_INVAL, "engine is NULL");
    if (select_budget < 1 || max_rounds < 1) return fail(PBB_E_INVAL, "limits must be >= 1");
    e->select_budget = select_budget;
    e->max_rounds = max_rounds;
    return PBB_OK;
}

int pbb_diag_sample_nodes(pbb_engine* e, int32_t capacity, int32_t rate_log2)
{
    if (!e) return fail(PBB_E_INVAL, "engine is NULL");
    if (capacity < 0 || rate_log2 < 0 || rate_log2 > 30) return fail(PBB_E_INVAL, "bad sampling parameters");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(cudaStreamSynchronize(e->st));
    cudaFree(e->sample_d);
    cudaFree(e->sample_rec);
    e->sample_d = nullptr;
    e->sample_rec = nullptr;
    e->group.sample = nullptr;
    if (capacity > 0) {
        e->sample_stride = PBB_SAMPLE_HDR + 5 * e->H.n;
        const size_t bytes = sizeof(int) * (size_t)capacity * e->sample_stride;
        CK(cudaMalloc(&e->sample_rec, bytes));
        CK(cudaMalloc(&e->sample_d, sizeof(SampleBuf)));
        CK(cudaMemsetAsync(e->sample_rec, 0, bytes, e->st));
        SampleBuf sb;
        sb.count = 0;
        sb.cap = (unsigned)capacity;
        sb.rate_mask = (1u << rate_log2) - 1u;
        sb.stride = e->sample_stride;
        sb.rec = e->sample_rec;
        CK(cudaMemcpyAsync(e->sample_d, &sb, sizeof(sb), cudaMemcpyHostToDevice, e->st));
        e->group.sample = e->sample_d;
    }
    CK(cudaMemcpyAsync(e->group_d, &e->group, sizeof(DevGroup), cudaMemcpyHostToDevice, e->st));
    CK(cudaStreamSynchronize(e->st));
    return PBB_OK;
}

int pbb_diag_get_samples(pbb_engine* e, int32_t max_records, int32_t* out, int32_t* count)
{
    if (!e || !count) return fail(PBB_E_INVAL, "NULL argument");
    *count = 0;
    if (!e->sample_d) return PBB_OK;
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(cudaStreamSynchronize(e->st));
    SampleBuf sb;
    CK(cudaMemcpy(&sb, e->sample_d, sizeof(sb), cudaMemcpyDeviceToHost));
    const int have = (int)std::min(sb.count, sb.cap);
    const int k = std::min(have, std::max(0, (int)max_records));
    if (k > 0) {
        if (!out) return fail(PBB_E_INVAL, "out is NULL");
        CK(cudaMemcpy(out, e->sample_rec, sizeof(int) * (size_t)k * e->sample_stride, cudaMemcpyDeviceToHost));
    }
    *count = max_records > 0 ? k : have;
    return PBB_OK;
}

int pbb_explore(pbb_engine* e, double seconds, int32_t* done)
{
    if (!e || !e->started) return fail(PBB_E_INVAL, "engine not started");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    int rc = settle(e);
    if (rc) return rc;
    if (!e->done) {
        // a launch never runs unbounded: at most 120 s of device time per window
        const double win = (seconds > 0 && seconds < 120.0) ? seconds : 120.0;
        const unsigned long long budget = (unsigned long long)(win * 1e9);
        CK(cudaEventRecord(e->ev0, e->st));
        int variant = e->sample_d ? 2 : ((e->cfg.sorted_dfs || e->cfg.early_stop_johnson) ? 1 : 0);
        // the fixed build also needs the per-warp masks in the launch
        const bool masks = e->smem == pbbl::smem_bytes(e->H.n, e->H.m, e->H.Ppad, e->warps, 1);
        if (variant == 0 && e->cfg.bounding_mode == 2 && e->cfg.branching_mode == 3 && !e->cfg.find_all && masks)
            variant = 3;
        CK(pbbl::launch_explore(e->nw, e->group_d, e->ngroups_d, e->ctas, e->warps, e->smem, budget, e->max_rounds,
                                e->select_budget, e->st, variant));
        CK(cudaEventRecord(e->ev1, e->st));
        rc = wait_event(e->ev1, e->wait_limit_s < 0 ? win + 60.0 : e->wait_limit_s);
        if (rc == PBB_E_TIMEOUT) {
            e->pending = true;
            return fail(PBB_E_TIMEOUT, "the exploration window did not end within the host wait limit; it ends by "
                                       "its own device-time budget and the next call accounts for it");
        }
        if (rc) return rc;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e->ev0, e->ev1));
        e->dev_seconds += ms * 1e-3;
        int active = 0;
        CK(cudaMemcpy(&active, &e->ctl->active, sizeof(int), cudaMemcpyDeviceToHost));
        e->done = (active == 0);
    }
    if (done) *done = e->done ? 1 : 0;
    return PBB_OK;
}

int pbb_get_result(pbb_engine* e, pbb_result* out)
{
    if (!e || !out) return fail(PBB_E_INVAL, "NULL argument");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(cudaStreamSynchronize(e->st));
    GroupCtl c;
    CK(cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof(*out));
    out->complete = e->done ? 1 : 0;
    const unsigned best_id = (unsigned)(c.best_key & 0xffffffffull);
    // a bound lowered from outside (pbb_set_ub) carries no permutation here
    out->found = (c.found > 0 && best_id != 0xffffffffu) ? 1 : 0;
    out->cost = (int32_t)(c.best_key >> 32);
    out->n_jobs = e->H.n;
    out->stats.decomposed = c.decomposed;
    out->stats.johnson_bounds = c.johnson_bounds;
    out->stats.simple_bounds = c.simple_bounds;
    out->stats.leaves = c.leaves;
    out->stats.steals = c.steals;
    out->device_seconds = e->dev_seconds;
    if (c.status & PBB_ST_BADINPUT) return fail(PBB_E_INVAL, "device reported bad input");
    if (out->found) {
        const unsigned id = (unsigned)(c.best_key & 0xffffffffull);
        if (id >= (unsigned)e->cfg.nb_ivms) return fail(PBB_E_CUDA, "corrupt best key");
        signed char buf[PBB_MAX_N];
        CK(cudaMemcpy(buf, e->bestperm + (size_t)id * PBB_MAX_N, PBB_MAX_N, cudaMemcpyDeviceToHost));
        for (int i = 0; i < e->H.n; i++) out->perm[i] = buf[i];
        out->has_perm = 1;
    } else if (e->from_neh && out->cost == e->ub) {
        // not improved: the NEH schedule the search started from
        int buf[PBB_MAX_N + 1];
        CK(cudaMemcpy(buf, e->neh_d, sizeof(buf), cudaMemcpyDeviceToHost));
        for (int i = 0; i < e->H.n; i++) out->perm[i] = buf[i];
        out->has_perm = 1;
    } else if ((int)e->start_perm.size() == e->H.n && out->cost == e->ub) {
        // not improved: the schedule that came with the starting bound
        for (int i = 0; i < e->H.n; i++) out->perm[i] = e->start_perm[i];
        out->has_perm = 1;
    }
    return PBB_OK;
}

int pbb_solve(pbb_engine* e, int32_t ub, const int32_t* root_perm, double time_limit_s, pbb_result* out)
{
    int rc = pbb_start(e, ub, root_perm);
    if (rc) return rc;
    int32_t done = e->done ? 1 : 0;
    while (!done) {
        double slice = e->slice_s;
        if (time_limit_s > 0) {
            const double left = time_limit_s - e->dev_seconds;
            if (left <= 0) break;
            slice = std::min(slice, left);
        }
        rc = pbb_explore(e, slice, &done);
        if (rc) return rc;
    }
    return pbb_get_result(e, out);
}

static int bound_children_impl(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t method,
                               int32_t count, const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                               int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                               int32_t* node_weak, int32_t* node_strong, int32_t* prio_begin = nullptr,
                               int32_t* prio_end = nullptr, int32_t* strong_idle = nullptr);

int pbb_bound_children(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t count,
                       const int32_t* sched, const int32_t* limit1, const int32_t* limit2, int32_t* weak_begin,
                       int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end, int32_t* node_weak,
                       int32_t* node_strong)
{
    return bound_children_impl(inst, johnson_mode, device, 0, count, sched, limit1, limit2, weak_begin, weak_end,
                               strong_begin, strong_end, node_weak, node_strong);
}

int pbb_bound_children_ex(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t count,
                          const int32_t* sched, const int32_t* limit1, const int32_t* limit2, const pbb_bound_out* out)
{
    if (!out) return fail(PBB_E_INVAL, "out is NULL");
    return bound_children_impl(inst, johnson_mode, device, 0, count, sched, limit1, limit2, out->weak_begin,
                               out->weak_end, out->strong_begin, out->strong_end, out->node_weak, out->node_strong,
                               out->prio_begin, out->prio_end, out->strong_idle);
}

int pbb_diag_bound_children(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t method,
                            int32_t count, const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                            int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                            int32_t* node_weak, int32_t* node_strong)
{
    if (method < 0 || method > 2)
        return fail(PBB_E_INVAL, "method must be 0 (sweeps), 1 (direct scans) or 2 (sweeps over free positions)");
    return bound_children_impl(inst, johnson_mode, device, method, count, sched, limit1, limit2, weak_begin,
                               weak_end, strong_begin, strong_end, node_weak, node_strong);
}

static int bound_children_impl(const pbb_instance* inst, int32_t johnson_mode, int32_t device, int32_t method,
                               int32_t count, const int32_t* sched, const int32_t* limit1, const int32_t* limit2,
                               int32_t* weak_begin, int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                               int32_t* node_weak, int32_t* node_strong, int32_t* prio_begin, int32_t* prio_end,
                               int32_t* strong_idle)
{
    if (count < 0 || (count > 0 && (!sched || !limit1 || !limit2))) return fail(PBB_E_INVAL, "bad node arrays");
    HostTables H;
    int rc = build_tables(inst, johnson_mode, H);
    if (rc) return rc;
    if (count == 0) return PBB_OK;
    const int n = H.n;
    for (int i = 0; i < count; i++) {
        if (limit1[i] < -1 || limit2[i] > n || limit1[i] >= limit2[i]) return fail(PBB_E_INVAL, "bad limits");
        std::vector<int> seen(n, 0);
        for (int t = 0; t < n; t++) {
            const int j = sched[(size_t)i * n + t];
            if (j < 0 || j >= n || seen[j]) return fail(PBB_E_INVAL, "schedule is not a permutation");
            seen[j] = 1;
        }
    }
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(device));
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    DeviceInstance di;
    rc = di.upload(H, st);
    int* buf = nullptr;
    unsigned* status = nullptr;
    const size_t cn = (size_t)count * n;
    const bool want_prio = prio_begin || prio_end;
    const size_t words = cn * 5 + (size_t)count * 4 + (want_prio ? 2 * cn : 0) + (strong_idle ? count : 0);
    do {
        if (rc) break;
        cudaError_t ce = cudaMalloc(&buf, sizeof(int) * words);
        if (ce == cudaSuccess) ce = cudaMalloc(&status, sizeof(unsigned));
        if (ce != cudaSuccess) { rc = cuda_fail(ce, "cudaMalloc"); break; }
        int* d_s = buf;
        int* d_wb = d_s + cn;
        int* d_we = d_wb + cn;
        int* d_sb = d_we + cn;
        int* d_se = d_sb + cn;
        int* d_l1 = d_se + cn;
        int* d_l2 = d_l1 + count;
        int* d_nw = d_l2 + count;
        int* d_ns = d_nw + count;
        BoundExtra X;
        int* tail = d_ns + count;
        if (want_prio) { X.prio_begin = tail; X.prio_end = tail + cn; tail += 2 * cn; }
        if (strong_idle) X.strong_idle = tail;
        cudaMemcpyAsync(d_s, sched, sizeof(int) * cn, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_l1, limit1, sizeof(int) * count, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_l2, limit2, sizeof(int) * count, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(status, 0, sizeof(unsigned), st);
        int smem = 0;
        const int warps = pick_warps(H, 8, device, smem);
        if (warps < 1) { rc = fail(PBB_E_INVAL, "instance tables do not fit in shared memory"); break; }
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        int ctas = (count + warps - 1) / warps;
        ctas = std::min(ctas, sms * 4);
        ce = pbbl::launch_bound(n <= 32 ? 1 : 2, di.view, count, d_s, d_l1, d_l2, d_wb, d_we, d_sb, d_se, d_nw, d_ns,
                                status, ctas, warps, smem, st, method, X);
        if (ce != cudaSuccess) { rc = cuda_fail(ce, "pbb_bound_kernel launch"); break; }
        if (weak_begin) cudaMemcpyAsync(weak_begin, d_wb, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (weak_end) cudaMemcpyAsync(weak_end, d_we, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (strong_begin) cudaMemcpyAsync(strong_begin, d_sb, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (strong_end) cudaMemcpyAsync(strong_end, d_se, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (node_weak) cudaMemcpyAsync(node_weak, d_nw, sizeof(int) * count, cudaMemcpyDeviceToHost, st);
        if (node_strong) cudaMemcpyAsync(node_strong, d_ns, sizeof(int) * count, cudaMemcpyDeviceToHost, st);
        if (prio_begin) cudaMemcpyAsync(prio_begin, X.prio_begin, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (prio_end) cudaMemcpyAsync(prio_end, X.prio_end, sizeof(int) * cn, cudaMemcpyDeviceToHost, st);
        if (strong_idle) cudaMemcpyAsync(strong_idle, X.strong_idle, sizeof(int) * count, cudaMemcpyDeviceToHost, st);
        unsigned hs = 0;
        cudaMemcpyAsync(&hs, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        ce = cudaStreamSynchronize(st);
        if (ce != cudaSuccess) { rc = cuda_fail(ce, "pbb_bound_kernel"); break; }
        if (hs & PBB_ST_BADINPUT) rc = fail(PBB_E_INVAL, "device rejected a node");
    } while (0);
    cudaFree(buf);
    cudaFree(status);
    di.release();
    cudaStreamDestroy(st);
    return rc;
}

int pbb_work_counters(pbb_engine* e, pbb_work* out)
{
    if (!e || !out) return fail(PBB_E_INVAL, "NULL argument");
    pbbh::DeviceGuard keep_callers_device;
    CK(cudaSetDevice(e->dev));
    {
        const int rs = settle(e);
        if (rs) return rs;
    }
    CK(cudaStreamSynchronize(e->st));
    GroupCtl c;
    CK(cudaMemcpy(&c, e->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    out->device_seconds = e->dev_seconds;
    out->n_jobs = e->H.n;
    out->n_machines = e->H.m;
    out->machine_pairs = e->H.P;
    out->decomposed = c.decomposed;
    out->simple_bounds = c.simple_bounds;
    out->johnson_bounds = c.johnson_bounds;
    out->johnson_sweeps = c.jsweeps;
    out->sweep_free_jobs = c.jfree;
    out->sweep_children = c.jchild;
    out->direct_children = c.jdirect;
    out->direct_free_jobs = c.jdirect_free;
    out->explorers = e->cfg.nb_ivms;
    out->warps = e->warps * e->ctas;
    out->status = (int32_t)c.status;
    return PBB_OK;
}

// NEH (heuristic/src/fastNEH.cpp:230-243 for the insertion procedure): jobs
// by decreasing total time (ties: lower id first); the first two keep the
// swapped order unless the original one is strictly better; each next job is
// inserted at the first position of least partial makespan.
int pbb_neh(const pbb_instance* inst, int32_t* perm, int32_t* cost)
{
    if (!inst || !inst->p || !perm) return fail(PBB_E_INVAL, "NULL argument");
    const int n = inst->n_jobs, m = inst->n_machines;
    if (n < 1 || m < 1) return fail(PBB_E_INVAL, "empty instance");
    const int32_t* p = inst->p;
    std::vector<int> tot(n, 0), order(n);
    for (int j = 0; j < n; j++) {
        for (int k = 0; k < m; k++) tot[j] += p[k * n + j];
        order[j] = j;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tot[a] > tot[b]; });
    std::vector<int> c(m);
    auto makespan = [&](const std::vector<int>& s) {
        std::fill(c.begin(), c.end(), 0);
        for (int j : s) {
            c[0] += p[j];
            for (int k = 1; k < m; k++) c[k] = std::max(c[k - 1], c[k]) + p[k * n + j];
        }
        return c[m - 1];
    };
    std::vector<int> seq;
    if (n == 1) {
        seq = {order[0]};
    } else {
        std::vector<int> a = {order[0], order[1]}, b = {order[1], order[0]};
        seq = makespan(a) < makespan(b) ? a : b;
        for (int k = 2; k < n; k++) {
            int best = INT_MAX, bpos = 0;
            std::vector<int> trial;
            for (int q = 0; q <= k; q++) {
                trial = seq;
                trial.insert(trial.begin() + q, order[k]);
                const int v = makespan(trial);
                if (v < best) { best = v; bpos = q; }
            }
            seq.insert(seq.begin() + bpos, order[k]);
        }
    }
    for (int i = 0; i < n; i++) perm[i] = seq[i];
    if (cost) *cost = makespan(seq);
    return PBB_OK;
}

}  // extern "C"
