// pbb_pool: many flow-shop instances resident on one GPU.  Each resident
// instance is a group (tables, explorers, queue, counters) of the same
// persistent explorer kernel the single-instance engine uses; one window
// launch explores all of them.  Between windows the host retires finished
// instances and admits queued ones by explorer-memory footprint, so requests
// that arrive while others run join the next window (continuous batching).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <deque>
#include <map>
#include <mutex>
#include <vector>

#include "pbb_types.h"
#include "pbb_devguard.h"
#include "pbb_launch.h"
#include "pbb_tables.h"
#include "pbb_heur.h"
#include "../../include/pbbperm.h"

namespace {

int pfail(int code, const char* msg)
{
    pbbh::set_error(msg);
    return code;
}

#define PCK(call, what)                               \
    do {                                              \
        cudaError_t e_ = (call);                      \
        if (e_ != cudaSuccess) {                      \
            pbbh::set_error(what);                    \
            return e_ == cudaErrorMemoryAllocation ? PBB_E_NOMEM : PBB_E_CUDA; \
        }                                             \
    } while (0)

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct Request {
    int64_t tag;
    std::vector<int32_t> root;
    pbb_config search;
    int32_t ub;
    pbbt::HostTables H;
};

struct Slot {
    bool used = false;
    int64_t tag = 0;
    int n = 0, m = 0;
    size_t off = 0, bytes = 0;      // explorer arena block
    int explorers = 0;
    int windows = 0;
    bool from_neh = false;          // started from the device NEH bound
    DevGroup g{};
};

// first-fit allocator over the explorer arena
struct Arena {
    std::map<size_t, size_t> free_blocks;   // offset -> size
    void init(size_t total) { free_blocks.clear(); free_blocks[0] = total; }
    bool alloc(size_t bytes, size_t& off)
    {
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
            if (it->second >= bytes) {
                off = it->first;
                const size_t rest = it->second - bytes;
                free_blocks.erase(it);
                if (rest) free_blocks[off + bytes] = rest;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        auto it = free_blocks.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_blocks.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_blocks.erase(next);
        }
        if (it != free_blocks.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_blocks.erase(it);
            }
        }
    }
};

}  // namespace

struct pbb_pool {
    pbb_pool_config cfg{};
    int dev = 0;
    cudaStream_t st = nullptr;
    int nw = 1, npad = 32, warps = 8, cpi = 1, epw = 1, smem = 0, root_smem = 0;
    int max_slots = 0;          // resident instances at most
    int grid = 0;               // CTAs of a window launch (all the CTAs of this shape the GPU holds)
    int tail_warps = 0, tail_grid = 0, tail_smem = 0;   // the tail's block shape (0 warps: none)
    int core_warps = PBB_CORE_WARPS, split_depth = PBB_SPLIT_DEPTH, share_after = PBB_SHARE_AFTER;
    int Ppad_max = 0;
    size_t table_stride = 0;
    size_t off_je = 0, off_p = 0, off_pm = 0, off_mt = 0, off_posj = 0;
    unsigned char* arena = nullptr;
    size_t arena_bytes = 0;
    unsigned char* tables = nullptr;
    GroupCtl* ctl = nullptr;
    GroupCtl* ctl_h = nullptr;  // pinned mirror, written by the window graph
    DevGroup* groups_d = nullptr;
    int* ngroups_d = nullptr;
    DevGroup* new_d = nullptr;
    int* ub_d = nullptr;
    int* roots_d = nullptr;
    int* ivals_d = nullptr;
    int* neh_d = nullptr;         // per slot: device NEH permutation [64] and makespan
    NehTask* neh_tasks_d = nullptr;
    cudaGraphExec_t window = nullptr;
    cudaGraphExec_t window_tail = nullptr;   // the same window with the tail's block shape
    cudaGraphExec_t window_fixed = nullptr, window_tail_fixed = nullptr;   // boundingMode 2 + MinMin builds
    bool masks = false, tail_masks = false;   // launches sized with the per-warp free-position masks
    std::vector<Slot> slots;
    // the FIFO and the finished results are shared with submitting and
    // polling threads; everything else belongs to the thread driving step()
    std::mutex mu;
    std::deque<Request> queue;
    std::vector<pbb_pool_result> done;
    Arena alloc;
    std::vector<int> pending_ub, pending_root;   // of the instances admitted in this step
    std::vector<NehTask> pending_neh;            // admitted instances that start from device NEH
};

extern "C" void pbb_pool_config_default(pbb_pool_config* c)
{
    if (!c) return;
    memset(c, 0, sizeof(*c));
    c->max_jobs = 32;
    c->max_machines = 20;
    c->warps_per_cta = 8;
    c->ctas_per_instance = 0;
    c->explorers_per_instance = 0;      // one explorer per warp slot of the grid
    c->window_s = 0.005;
    c->explorer_bytes = (int64_t)8 << 30;
}

extern "C" int pbb_pool_destroy(pbb_pool* P)
{
    if (!P) return PBB_OK;
    pbbh::DeviceGuard keep_callers_device;
    cudaSetDevice(P->dev);
    if (P->st) cudaStreamSynchronize(P->st);
    if (P->window) cudaGraphExecDestroy(P->window);
    if (P->window_tail) cudaGraphExecDestroy(P->window_tail);
    if (P->window_fixed) cudaGraphExecDestroy(P->window_fixed);
    if (P->window_tail_fixed) cudaGraphExecDestroy(P->window_tail_fixed);
    cudaFree(P->arena);
    cudaFree(P->tables);
    cudaFree(P->ctl);
    cudaFreeHost(P->ctl_h);
    cudaFree(P->groups_d);
    cudaFree(P->ngroups_d);
    cudaFree(P->new_d);
    cudaFree(P->ub_d);
    cudaFree(P->roots_d);
    cudaFree(P->ivals_d);
    cudaFree(P->neh_d);
    cudaFree(P->neh_tasks_d);
    if (P->st) cudaStreamDestroy(P->st);
    delete P;
    return PBB_OK;
}

namespace {

size_t explorer_block_bytes(int E, int npad)
{
    size_t b = align256((size_t)E * npad * npad);     // mat
    b += 5 * align256((size_t)E * npad);              // pos end dir pj bestperm
    b += 5 * align256((size_t)E * 4);                 // line state bestcost qseq qval
    b += align256((size_t)E * npad * PBB_PATH_INTS * 4);   // path levels
    return b;
}

void carve_explorers(unsigned char* base, int E, int npad, DevIvms& V)
{
    size_t o = 0;
    V.count = E;
    V.npad = npad;
    V.mat = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad * npad);
    V.pos = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad);
    V.end = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad);
    V.dir = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad);
    V.pj = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad);
    V.bestperm = reinterpret_cast<signed char*>(base + o); o += align256((size_t)E * npad);
    V.line = reinterpret_cast<int*>(base + o); o += align256((size_t)E * 4);
    V.state = reinterpret_cast<int*>(base + o); o += align256((size_t)E * 4);
    V.bestcost = reinterpret_cast<int*>(base + o); o += align256((size_t)E * 4);
    V.qseq = reinterpret_cast<unsigned*>(base + o); o += align256((size_t)E * 4);
    V.qval = reinterpret_cast<int*>(base + o); o += align256((size_t)E * 4);
    V.path = reinterpret_cast<int*>(base + o);
}

int pool_create(const pbb_pool_config* in, pbb_pool* P)
{
    pbb_pool_config c;
    pbb_pool_config_default(&c);
    if (in) {
        c = *in;
        pbb_pool_config d;
        pbb_pool_config_default(&d);
        if (c.warps_per_cta <= 0) c.warps_per_cta = d.warps_per_cta;
        if (c.ctas_per_instance < 0) c.ctas_per_instance = 0;
        if (c.explorers_per_instance < 0) c.explorers_per_instance = 0;
        if (c.window_s <= 0) c.window_s = d.window_s;
        if (c.explorer_bytes <= 0) c.explorer_bytes = d.explorer_bytes;
    }
    if (c.max_jobs < 2 || c.max_jobs > PBB_MAX_JOBS) return pfail(PBB_E_INVAL, "max_jobs must be in [2, 64]");
    if (c.max_machines < 2 || c.max_machines > PBB_MAX_MACHINES)
        return pfail(PBB_E_INVAL, "max_machines must be in [2, 32]");
    if (c.warps_per_cta > PBB_WARPS_MAX) return pfail(PBB_E_INVAL, "warps_per_cta must be <= 20");
    if (c.window_s > 120.0) return pfail(PBB_E_INVAL, "window_s must be <= 120");
    P->cfg = c;
    P->dev = c.device;
    pbbh::DeviceGuard keep_callers_device;
    PCK(cudaSetDevice(P->dev), "cudaSetDevice failed");
    PCK(cudaStreamCreateWithFlags(&P->st, cudaStreamNonBlocking), "stream creation failed");
    P->nw = c.max_jobs <= 32 ? 1 : 2;
    P->npad = 32 * P->nw;
    P->warps = c.warps_per_cta;
    P->cpi = c.ctas_per_instance;
    P->epw = c.explorers_per_instance;
    P->core_warps = c.core_warps > 0 ? c.core_warps : PBB_CORE_WARPS;
    P->split_depth = c.split_depth > 0 ? c.split_depth : PBB_SPLIT_DEPTH;
    P->share_after = c.share_after > 0 ? c.share_after : (c.share_after < 0 ? 0 : PBB_SHARE_AFTER);
    const int Pmax = c.max_machines * (c.max_machines - 1) / 2;
    P->Ppad_max = (Pmax + 31) / 32 * 32;
    P->smem = pbbl::smem_bytes(c.max_jobs, c.max_machines, P->Ppad_max, P->warps);
    P->root_smem = pbbl::smem_bytes(c.max_jobs, c.max_machines, P->Ppad_max, 1);
    int optin = 0, sms = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, P->dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->dev);
    if (P->smem > optin) return pfail(PBB_E_INVAL, "tables of max_jobs x max_machines do not fit in shared memory");
    int per_sm = pbbl::explore_ctas_per_sm(P->nw, P->warps, P->smem);
    if (per_sm < 1) return pfail(PBB_E_INVAL, "explorer kernel cannot be resident with this block shape");
    {
        // per-warp free-position masks, when they cost no resident CTA
        const int ms = pbbl::smem_bytes(c.max_jobs, c.max_machines, P->Ppad_max, P->warps, 1);
        if (ms <= optin && pbbl::explore_ctas_per_sm(P->nw, P->warps, ms) >= per_sm) {
            P->smem = ms;
            P->masks = true;
        }
    }
    // every window launches all the CTAs the GPU holds at once and spreads
    // them over the resident instances
    int capacity = sms * per_sm;
    if (capacity < 1) capacity = 1;
    P->grid = capacity;
    // the tail's block shape: wider CTAs once few instances remain (the heavy
    // searches that finish last want every warp an SM holds)
    const int tw = c.tail_warps == 0 ? PBB_WARPS_MAX : c.tail_warps;
    if (tw > P->warps && tw <= PBB_WARPS_MAX) {
        int ts = pbbl::smem_bytes(c.max_jobs, c.max_machines, P->Ppad_max, tw);
        const int tper = ts <= optin ? pbbl::explore_ctas_per_sm(P->nw, tw, ts) : 0;
        const int tms = pbbl::smem_bytes(c.max_jobs, c.max_machines, P->Ppad_max, tw, 1);
        bool tm = false;
        if (tper >= 1 && tms <= optin && pbbl::explore_ctas_per_sm(P->nw, tw, tms) >= tper) {
            ts = tms;
            tm = true;
        }
        if (tper >= 1) {
            P->tail_warps = tw;
            P->tail_smem = ts;
            P->tail_grid = sms * tper;
            P->tail_masks = tm;
        }
    }
    // default explorer count: every warp of the widest grid owns one, so that
    // an instance left alone at the end of a batch can keep the whole GPU busy
    if (P->epw <= 0) P->epw = std::max(P->grid * P->warps, P->tail_grid * P->tail_warps);
    P->max_slots = c.max_resident > 0 ? std::min(c.max_resident, capacity) : capacity;
    // per-slot instance tables
    P->off_je = 0;
    P->off_p = align256(P->off_je + (size_t)c.max_jobs * P->Ppad_max * 8);
    P->off_pm = align256(P->off_p + (size_t)c.max_jobs * c.max_machines * 4);
    P->off_mt = align256(P->off_pm + 2 * (size_t)P->Ppad_max);
    P->off_posj = align256(P->off_mt + 2 * (size_t)c.max_machines * 4);
    P->table_stride = align256(P->off_posj + (size_t)c.max_jobs * P->Ppad_max);
    const int S = P->max_slots;
    PCK(cudaMalloc(&P->tables, P->table_stride * S), "table memory");
    PCK(cudaMalloc(&P->ctl, sizeof(GroupCtl) * S), "control blocks");
    PCK(cudaMemset(P->ctl, 0, sizeof(GroupCtl) * S), "control blocks");
    PCK(cudaMallocHost(&P->ctl_h, sizeof(GroupCtl) * S), "pinned control mirror");
    memset(P->ctl_h, 0, sizeof(GroupCtl) * S);
    PCK(cudaMalloc(&P->groups_d, sizeof(DevGroup) * S), "group list");
    PCK(cudaMalloc(&P->new_d, sizeof(DevGroup) * S), "group list");
    PCK(cudaMalloc(&P->ngroups_d, sizeof(int)), "group count");
    PCK(cudaMemset(P->ngroups_d, 0, sizeof(int)), "group count");
    PCK(cudaMalloc(&P->ub_d, sizeof(int) * S), "bounds");
    PCK(cudaMalloc(&P->roots_d, sizeof(int) * S * PBB_MAX_N), "roots");
    PCK(cudaMalloc(&P->ivals_d, sizeof(int) * S * 2 * PBB_MAX_N), "intervals");
    PCK(cudaMalloc(&P->neh_d, sizeof(int) * S * (PBB_MAX_N + 1)), "heuristic results");
    PCK(cudaMalloc(&P->neh_tasks_d, sizeof(NehTask) * S), "heuristic tasks");
    P->arena_bytes = (size_t)c.explorer_bytes;
    const int E = P->epw;
    if (explorer_block_bytes(E, P->npad) > P->arena_bytes)
        return pfail(PBB_E_INVAL, "explorer_bytes is smaller than one instance's footprint");
    PCK(cudaMalloc(&P->arena, P->arena_bytes), "explorer memory");
    P->alloc.init(P->arena_bytes);
    P->slots.assign(S, Slot());
    // the window: explorer kernel and control read-back, as one graph; one
    // graph per block shape (bulk, tail) and explorer build (the general one,
    // and the one with boundingMode 2 and MinMin compiled in, used while every
    // resident instance searches that way)
    const unsigned long long budget = (unsigned long long)(c.window_s * 1e9);
    // the tail's windows last at least 20 ms: its few long searches gain
    // nothing from frequent admissions
    const unsigned long long tail_budget = std::max(budget, 20000000ull);
    auto capture = [&](int grid, int warps, int smem, unsigned long long win, int variant,
                       cudaGraphExec_t* out) -> int {
        cudaGraph_t graph = nullptr;
        PCK(cudaStreamBeginCapture(P->st, cudaStreamCaptureModeRelaxed), "graph capture");
        cudaError_t e1 = pbbl::launch_explore(P->nw, P->groups_d, P->ngroups_d, grid, warps, smem, win, INT_MAX, 4096,
                                              P->st, variant);
        cudaError_t e3 = cudaMemcpyAsync(P->ctl_h, P->ctl, sizeof(GroupCtl) * P->slots.size(),
                                         cudaMemcpyDeviceToHost, P->st);
        cudaError_t e4 = cudaStreamEndCapture(P->st, &graph);
        if (e1 || e3 || e4) {
            if (graph) cudaGraphDestroy(graph);
            return pfail(PBB_E_CUDA, "capturing a window graph failed");
        }
        cudaError_t e5 = cudaGraphInstantiate(out, graph, 0);
        cudaGraphDestroy(graph);
        if (e5) return pfail(PBB_E_CUDA, "instantiating a window graph failed");
        return PBB_OK;
    };
    int rc = capture(P->grid, P->warps, P->smem, budget, 0, &P->window);
    if (!rc && P->masks) rc = capture(P->grid, P->warps, P->smem, budget, 3, &P->window_fixed);
    if (!rc && P->tail_warps > 0) {
        rc = capture(P->tail_grid, P->tail_warps, P->tail_smem, tail_budget, 0, &P->window_tail);
        if (!rc && P->tail_masks)
            rc = capture(P->tail_grid, P->tail_warps, P->tail_smem, tail_budget, 3, &P->window_tail_fixed);
    }
    if (rc) return rc;
    return PBB_OK;
}

}  // namespace

extern "C" int pbb_pool_create(const pbb_pool_config* cfg, pbb_pool** out)
{
    if (!out) return pfail(PBB_E_INVAL, "out is NULL");
    *out = nullptr;
    pbb_pool* P = new pbb_pool();
    const int rc = pool_create(cfg, P);
    if (rc) {
        pbb_pool_destroy(P);
        return rc;
    }
    *out = P;
    return PBB_OK;
}

extern "C" int pbb_pool_submit(pbb_pool* P, const pbb_instance* inst, const pbb_config* search, int32_t ub,
                               const int32_t* root_perm, int64_t tag)
{
    if (!P) return pfail(PBB_E_INVAL, "pool is NULL");
    if (!inst || !inst->p) return pfail(PBB_E_INVAL, "instance is NULL");
    if (inst->n_jobs > P->cfg.max_jobs || inst->n_machines > P->cfg.max_machines)
        return pfail(PBB_E_INVAL, "instance larger than the pool's max_jobs x max_machines");
    if (ub < 0 && ub != PBB_UB_NEH) return pfail(PBB_E_INVAL, "ub must be >= 0 (or PBB_UB_NEH)");
    Request r;
    r.tag = tag;
    pbb_config_default(&r.search);
    if (search) r.search = *search;
    const pbb_config& c = r.search;
    const int rs = pbbh::check_search(&c);
    if (rs) return rs;
    if (c.sorted_dfs)
        return pfail(PBB_E_UNSUPPORTED, "the pool explores with sortedDFS = 0 (the single-instance engine takes 1)");
    const int rc = pbbt::build_tables(inst, c.johnson_mode, r.H);
    if (rc) return rc;
    const int n = inst->n_jobs;
    r.root.assign(PBB_MAX_N, 0);
    std::vector<int> seen(n, 0);
    for (int i = 0; i < n; i++) {
        const int j = root_perm ? root_perm[i] : i;
        if (j < 0 || j >= n || seen[j]) return pfail(PBB_E_INVAL, "root_perm is not a permutation of 0..n-1");
        seen[j] = 1;
        r.root[i] = j;
    }
    r.ub = ub;
    std::lock_guard<std::mutex> lock(P->mu);
    P->queue.push_back(std::move(r));
    return PBB_OK;
}

namespace {

// admit queued instances while a slot and explorer memory are free (FIFO);
// submitters may push concurrently, so each request is moved out under the lock
int admit(pbb_pool* P, std::vector<int>& admitted)
{
    const int E = P->epw;
    const size_t bytes = explorer_block_bytes(E, P->npad);
    while (true) {
        int s = -1;
        for (int i = 0; i < P->max_slots; i++)
            if (!P->slots[i].used) { s = i; break; }
        if (s < 0) break;
        size_t off = 0;
        if (!P->alloc.alloc(bytes, off)) break;
        Request r;
        {
            std::lock_guard<std::mutex> lock(P->mu);
            if (P->queue.empty()) {
                P->alloc.release(off, bytes);
                break;
            }
            r = std::move(P->queue.front());
            P->queue.pop_front();
        }
        const pbbt::HostTables& H = r.H;
        unsigned char* tb = P->tables + (size_t)s * P->table_stride;
        PCK(cudaMemcpyAsync(tb + P->off_je, H.je.data(), H.je.size() * 8, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(tb + P->off_p, H.p.data(), H.p.size() * 4, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(tb + P->off_pm, H.pm0.data(), H.Ppad, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(tb + P->off_pm + H.Ppad, H.pm1.data(), H.Ppad, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(tb + P->off_mt, H.min_arr.data(), H.m * 4, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(tb + P->off_mt + H.m * 4, H.min_dep.data(), H.m * 4, cudaMemcpyHostToDevice, P->st),
            "upload");
        PCK(cudaMemcpyAsync(tb + P->off_posj, H.posj.data(), H.posj.size(), cudaMemcpyHostToDevice, P->st), "upload");
        Slot& sl = P->slots[s];
        sl = Slot();
        sl.used = true;
        sl.tag = r.tag;
        sl.n = H.n;
        sl.m = H.m;
        sl.off = off;
        sl.bytes = bytes;
        sl.explorers = E;
        DevGroup& g = sl.g;
        g.inst.n = H.n; g.inst.m = H.m; g.inst.P = H.P; g.inst.Ppad = H.Ppad;
        g.inst.p = reinterpret_cast<const int*>(tb + P->off_p);
        g.inst.je = reinterpret_cast<const unsigned long long*>(tb + P->off_je);
        g.inst.pm0 = tb + P->off_pm;
        g.inst.pm1 = tb + P->off_pm + H.Ppad;
        g.inst.min_arr = reinterpret_cast<const int*>(tb + P->off_mt);
        g.inst.min_dep = reinterpret_cast<const int*>(tb + P->off_mt + H.m * 4);
        g.inst.posj = tb + P->off_posj;
        g.search.bound_mode = r.search.bounding_mode;
        g.search.branch_mode = r.search.branching_mode;
        g.search.find_all = r.search.find_all ? 1 : 0;
        g.search.sort_nodes = r.search.sorted_dfs;
        g.search.sort_crit = r.search.sorting_criterion;
        // the pool's window graph runs the default explorer, which has no early
        // Johnson exit: it leaves every decision unchanged, so it is not needed
        g.search.early_stop = 0;
        g.search.core_warps = P->core_warps;
        g.search.split_depth = P->split_depth;
        g.search.share_after = P->share_after;
        carve_explorers(P->arena + off, E, P->npad, g.ivm);
        g.ctl = P->ctl + s;
        admitted.push_back(s);
        P->pending_ub.push_back(r.ub);
        sl.from_neh = r.ub == PBB_UB_NEH;
        if (sl.from_neh) {
            // device NEH at admission: its makespan lands in this admission's
            // bound slot before the reset kernel reads it
            NehTask t;
            t.p = g.inst.p;
            t.n = H.n;
            t.m = H.m;
            t.perm = P->neh_d + (size_t)s * (PBB_MAX_N + 1);
            t.cost = t.perm + PBB_MAX_N;
            t.ub = P->ub_d + (P->pending_ub.size() - 1);
            P->pending_neh.push_back(t);
        }
        P->pending_root.insert(P->pending_root.end(), r.root.begin(), r.root.end());
    }
    return PBB_OK;
}

}  // namespace

extern "C" int pbb_pool_step(pbb_pool* P, int32_t* resident, int32_t* queued)
{
    if (!P) return pfail(PBB_E_INVAL, "pool is NULL");
    pbbh::DeviceGuard keep_callers_device;
    PCK(cudaSetDevice(P->dev), "cudaSetDevice failed");
    std::vector<int> admitted;
    P->pending_ub.clear();
    P->pending_root.clear();
    P->pending_neh.clear();
    int rc = admit(P, admitted);
    if (rc) return rc;
    const int na = (int)admitted.size();
    if (na > 0) {
        // empty explorers, reset counters, bound the roots of the newcomers
        std::vector<DevGroup> ng(na);
        std::vector<int> iv((size_t)na * 2 * PBB_MAX_N, 0);
        for (int i = 0; i < na; i++) {
            const Slot& sl = P->slots[admitted[i]];
            ng[i] = sl.g;
            for (int e = 0; e < sl.n; e++) {
                iv[(size_t)(2 * i) * PBB_MAX_N + e] = 0;
                iv[(size_t)(2 * i + 1) * PBB_MAX_N + e] = sl.n - 1 - e;
            }
        }
        PCK(cudaMemcpyAsync(P->new_d, ng.data(), sizeof(DevGroup) * na, cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(P->ub_d, P->pending_ub.data(), sizeof(int) * na, cudaMemcpyHostToDevice, P->st),
            "upload");
        PCK(cudaMemcpyAsync(P->roots_d, P->pending_root.data(), sizeof(int) * na * PBB_MAX_N,
                            cudaMemcpyHostToDevice, P->st), "upload");
        PCK(cudaMemcpyAsync(P->ivals_d, iv.data(), sizeof(int) * iv.size(), cudaMemcpyHostToDevice, P->st),
            "upload");
        if (!P->pending_neh.empty()) {
            const int nn = (int)P->pending_neh.size();
            PCK(cudaMemcpyAsync(P->neh_tasks_d, P->pending_neh.data(), sizeof(NehTask) * nn, cudaMemcpyHostToDevice,
                                P->st), "upload");
            PCK(pbbl::launch_neh(P->neh_tasks_d, nn, P->st), "heuristic launch");
        }
        PCK(pbbl::launch_reset(P->new_d, na, P->ub_d, P->st), "reset launch");
        PCK(pbbl::launch_root(P->nw, P->new_d, na, P->roots_d, P->ivals_d, PBB_MAX_N, P->root_smem, P->st),
            "root launch");
    }
    // the window over every resident instance
    std::vector<DevGroup> act;
    std::vector<int> act_slot;
    for (int s = 0; s < P->max_slots; s++) {
        if (!P->slots[s].used) continue;
        act.push_back(P->slots[s].g);
        act_slot.push_back(s);
    }
    // the tail: nothing waits and few instances remain -- wide CTAs, at least
    // four per resident instance
    bool waiting;
    {
        std::lock_guard<std::mutex> lock(P->mu);
        waiting = !P->queue.empty();
    }
    const bool tail = P->tail_warps > 0 && !waiting && (int)act.size() * 4 <= P->tail_grid;
    const int grid = tail ? P->tail_grid : P->grid;
    {
        // all resident CTAs, spread evenly (a lone instance in the tail of a
        // batch gets the whole GPU), capped by ctas_per_instance when set
        const int na = (int)act.size();
        int first = 0;
        for (int i = 0; i < na; i++) {
            int c = grid / std::max(1, na) + (i < grid % std::max(1, na) ? 1 : 0);
            if (P->cpi > 0 && c > P->cpi) c = P->cpi;
            if (c < 1) c = 1;
            act[i].first_cta = first;
            act[i].ctas = c;
            first += c;
        }
    }
    const int nact = (int)act.size();
    if (nact > 0) {
        PCK(cudaMemcpyAsync(P->groups_d, act.data(), sizeof(DevGroup) * nact, cudaMemcpyHostToDevice, P->st),
            "upload");
    }
    PCK(cudaMemcpyAsync(P->ngroups_d, &nact, sizeof(int), cudaMemcpyHostToDevice, P->st), "upload");
    bool fixed = true;
    for (int i = 0; i < nact; i++)
        fixed = fixed && act[i].search.bound_mode == 2 && act[i].search.branch_mode == 3 && !act[i].search.find_all &&
                act[i].inst.posj != nullptr;
    cudaGraphExec_t win = tail ? P->window_tail : P->window;
    if (fixed && tail && P->window_tail_fixed) win = P->window_tail_fixed;
    if (fixed && !tail && P->window_fixed) win = P->window_fixed;
    if (nact > 0) PCK(cudaGraphLaunch(win, P->st), "window launch");
    PCK(cudaStreamSynchronize(P->st), "window");
    // retire the finished instances
    for (int i = 0; i < nact; i++) {
        const int s = act_slot[i];
        Slot& sl = P->slots[s];
        sl.windows++;
        const GroupCtl& c = P->ctl_h[s];
        if (c.active != 0) continue;
        pbb_pool_result pr;
        memset(&pr, 0, sizeof(pr));
        pr.tag = sl.tag;
        pr.windows = sl.windows;
        pr.status = (c.status & PBB_ST_BADINPUT) ? PBB_E_INVAL : PBB_OK;
        pbb_result& r = pr.result;
        const unsigned id = (unsigned)(c.best_key & 0xffffffffull);
        // an instance the device flagged is neither complete nor solved
        const bool ok = pr.status == PBB_OK;
        r.complete = ok ? 1 : 0;
        r.found = (ok && c.found > 0 && id != 0xffffffffu && id < (unsigned)sl.explorers) ? 1 : 0;
        r.cost = (int32_t)(c.best_key >> 32);
        r.n_jobs = sl.n;
        r.stats.decomposed = c.decomposed;
        r.stats.johnson_bounds = c.johnson_bounds;
        r.stats.simple_bounds = c.simple_bounds;
        r.stats.leaves = c.leaves;
        r.stats.steals = c.steals;
        if (r.found) {
            signed char buf[PBB_MAX_N];
            PCK(cudaMemcpy(buf, sl.g.ivm.bestperm + (size_t)id * sl.g.ivm.npad, sl.n, cudaMemcpyDeviceToHost),
                "result read-back");
            for (int j = 0; j < sl.n; j++) r.perm[j] = buf[j];
            r.has_perm = 1;
        } else if (ok && sl.from_neh) {
            // not improved: the device NEH schedule is optimal
            int buf[PBB_MAX_N + 1];
            PCK(cudaMemcpy(buf, P->neh_d + (size_t)s * (PBB_MAX_N + 1), sizeof(buf), cudaMemcpyDeviceToHost),
                "result read-back");
            for (int j = 0; j < sl.n; j++) r.perm[j] = buf[j];
            r.has_perm = buf[PBB_MAX_N] == r.cost ? 1 : 0;
        }
        {
            std::lock_guard<std::mutex> lock(P->mu);
            P->done.push_back(pr);
        }
        P->alloc.release(sl.off, sl.bytes);
        sl = Slot();
    }
    int res = 0;
    for (int s = 0; s < P->max_slots; s++) res += P->slots[s].used ? 1 : 0;
    if (resident) *resident = res;
    if (queued) {
        std::lock_guard<std::mutex> lock(P->mu);
        *queued = (int32_t)P->queue.size();
    }
    return PBB_OK;
}

extern "C" int pbb_pool_poll(pbb_pool* P, pbb_pool_result* out, int32_t max, int32_t* count)
{
    if (!P || (!out && max > 0)) return pfail(PBB_E_INVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(P->mu);
    const int k = std::min((int)P->done.size(), (int)std::max(0, max));
    for (int i = 0; i < k; i++) out[i] = P->done[i];
    P->done.erase(P->done.begin(), P->done.begin() + k);
    if (count) *count = k;
    return PBB_OK;
}

extern "C" int pbb_batch_solve(const pbb_instance* inst, int32_t count, const pbb_config* search, const int32_t* ubs,
                               const pbb_pool_config* pool_cfg, pbb_result* results)
{
    if (count < 0 || (count > 0 && (!inst || !results))) return pfail(PBB_E_INVAL, "bad arguments");
    if (count == 0) return PBB_OK;
    pbb_pool_config c;
    if (pool_cfg) {
        c = *pool_cfg;
    } else {
        pbb_pool_config_default(&c);
        c.max_jobs = 2;
        c.max_machines = 2;
        for (int i = 0; i < count; i++) {
            c.max_jobs = std::max(c.max_jobs, (int32_t)inst[i].n_jobs);
            c.max_machines = std::max(c.max_machines, (int32_t)inst[i].n_machines);
        }
        c.window_s = 0.02;
    }
    pbb_pool* P = nullptr;
    int rc = pbb_pool_create(&c, &P);
    if (rc) return rc;
    // The whole batch is known: admit the largest instances first (jobs, then
    // machines), so that the long searches start early and overlap with the
    // many short ones instead of forming a tail after them.  Results are
    // matched back by tag, so the order is invisible to the caller.
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        if (inst[a].n_jobs != inst[b].n_jobs) return inst[a].n_jobs > inst[b].n_jobs;
        return inst[a].n_machines > inst[b].n_machines;
    });
    for (int q0 = 0; q0 < count && !rc; q0++) {
        const int i = order[q0];
        rc = pbb_pool_submit(P, &inst[i], search, ubs ? ubs[i] : INT32_MAX, nullptr, i);
    }
    int32_t res = 0, q = count;
    std::vector<pbb_pool_result> out(count);
    int got_total = 0;
    int first_bad = PBB_OK;     // first per-instance error, returned after the batch
    while (!rc && (res > 0 || q > 0 || got_total < count)) {
        rc = pbb_pool_step(P, &res, &q);
        if (rc) break;
        int32_t got = 0;
        rc = pbb_pool_poll(P, out.data(), count, &got);
        for (int i = 0; i < got; i++) {
            const int64_t t = out[i].tag;
            if (t >= 0 && t < count) results[t] = out[i].result;
            if (out[i].status != PBB_OK && first_bad == PBB_OK) first_bad = out[i].status;
        }
        got_total += got;
        if (res == 0 && q == 0) break;
    }
    pbb_pool_destroy(P);
    if (!rc && first_bad != PBB_OK) return pfail(first_bad, "the device rejected an instance of the batch");
    return rc;
}
