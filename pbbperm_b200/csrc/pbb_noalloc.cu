// pbb_bound_children_noalloc: the batched children-bound entry point for
// callers that cannot allocate GPU memory -- code that runs inside another
// framework's memory pool, a plugin handed only device buffers, or a process
// whose allocator is owned elsewhere.  Inputs and outputs are the caller's
// device buffers; the kernel's only scratch (the instance's Johnson / weak
// bound tables and a status word) lives in the file-scope device array below,
// so the call makes no cudaMalloc, cudaFree, or other allocating call.
//
// Limits and behaviour, for a user of this library:
//   * the scratch array is PBB_NOALLOC_SCRATCH_BYTES (112 KiB) on every GPU
//     that loads the library, held until the process exits; it fits instances
//     of at most 64 jobs and 20 machines (190 machine pairs) -- larger ones are
//     rejected with PBB_E_INVAL;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   * every call reuses the same array and leaves its tables in it; the status
//     word is cleared at the start of each call.  Calls whose work overlaps on
//     the GPU (other host threads, other streams) race on the array and must
//     not be issued concurrently; this entry point serialises its own host
//     callers and waits for its stream before returning;
//   * the calling thread's current device is the same after the call as
//     before it (the call selects `device` only while it runs);
//   * the block shape shrinks (8 warps down to 1) until the tables fit the
//     device's per-block shared memory; if even one warp does not fit, the
//     call returns PBB_E_INVAL.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <climits>
#include <mutex>

#include "pbb_types.h"
#include "pbb_launch.h"
#include "pbb_tables.h"
#include "pbb_devguard.h"
#include "../../include/pbbperm.h"

#define PBB_NOALLOC_MAX_N 64
#define PBB_NOALLOC_MAX_M 20
#define PBB_NOALLOC_MAX_PPAD 192   // 190 pairs rounded up to 32
#define PBB_NOALLOC_SCRATCH_BYTES (112 * 1024)
#define PBB_NOALLOC_MAX_DEVICES 64

// scratch layout (byte offsets, each 256-aligned)
#define NA_STATUS_OFF 0
#define NA_JE_OFF 256
#define NA_JE_BYTES (PBB_NOALLOC_MAX_N * PBB_NOALLOC_MAX_PPAD * 8)
#define NA_P_OFF (NA_JE_OFF + NA_JE_BYTES)
#define NA_P_BYTES (PBB_NOALLOC_MAX_N * PBB_NOALLOC_MAX_M * 4)
#define NA_PM_OFF (NA_P_OFF + NA_P_BYTES)
#define NA_PM_BYTES 512
#define NA_MT_OFF (NA_PM_OFF + NA_PM_BYTES)
#define NA_MT_BYTES 256
#define NA_END (NA_MT_OFF + NA_MT_BYTES)

static_assert(NA_END <= PBB_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout exceeds its array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[PBB_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mutex;
unsigned char* g_scratch_addr[PBB_NOALLOC_MAX_DEVICES];   // device address of the array, per device
int g_smem_optin[PBB_NOALLOC_MAX_DEVICES];                 // per-block shared memory limit, per device

// Host staging of the tables (static: building them allocates nothing).
struct StagedTables {
    unsigned long long je[PBB_NOALLOC_MAX_N * PBB_NOALLOC_MAX_PPAD];
    int p[PBB_NOALLOC_MAX_N * PBB_NOALLOC_MAX_M];
    unsigned char pm[2 * PBB_NOALLOC_MAX_PPAD];
    int mt[2 * PBB_NOALLOC_MAX_M];
};
StagedTables g_stage;

}  // namespace

static int na_fail(int code, const char* msg)
{
    pbbh::set_error(msg);
    return code;
}

// Tables of the instance into the static host staging area, with the same
// builder (and so the same Johnson tie order) as the allocating entry points.
static int na_build_tables(const pbb_instance* inst, int johnson_mode, int& P, int& Ppad)
{
    const int n = inst->n_jobs, m = inst->n_machines;
    const int rc = pbbt::check_times(inst->p, n, m);
    if (rc != PBB_OK) return rc;
    memcpy(g_stage.p, inst->p, sizeof(int) * n * m);
    P = pbbt::count_pairs(m, johnson_mode);
    Ppad = (P + 31) / 32 * 32;
    pbbt::TableSpans T{g_stage.je, nullptr, g_stage.pm, g_stage.pm + Ppad, g_stage.mt, g_stage.mt + m};
    pbbt::fill_tables(inst->p, n, m, johnson_mode, Ppad, T);
    return PBB_OK;
}

// Every node must be a permutation of 0..n-1 with -1 <= limit1 < limit2 <= n;
// a failure sets the status word (the bound kernel then is not launched).
__global__ void pbb_noalloc_check_kernel(int n, int count, const int* sched, const int* l1, const int* l2)
{
    unsigned* status = reinterpret_cast<unsigned*>(g_noalloc_scratch + NA_STATUS_OFF);
    for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < count; node += gridDim.x * blockDim.x) {
        bool ok = l1[node] >= -1 && l2[node] <= n && l1[node] < l2[node];
        unsigned long long seen = 0ull;
        for (int i = 0; i < n && ok; i++) {
            const int j = sched[(size_t)node * n + i];
            if (j < 0 || j >= n || ((seen >> j) & 1ull)) ok = false;
            else seen |= 1ull << j;
        }
        if (!ok) atomicOr(status, PBB_ST_BADINPUT);
    }
}

#define NA_CK(call, what)                                                \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) {                                         \
            pbbh::set_error(what);                                       \
            return PBB_E_CUDA;                                           \
        }                                                                \
    } while (0)

extern "C" int pbb_bound_children_noalloc(const pbb_instance* inst, int32_t johnson_mode, int32_t device,
                                          void* stream, int32_t count, const int32_t* sched,
                                          const int32_t* limit1, const int32_t* limit2, int32_t* weak_begin,
                                          int32_t* weak_end, int32_t* strong_begin, int32_t* strong_end,
                                          int32_t* node_weak, int32_t* node_strong)
{
    std::lock_guard<std::mutex> guard(g_noalloc_mutex);
    if (!inst || !inst->p) return na_fail(PBB_E_INVAL, "instance is NULL");
    const int n = inst->n_jobs, m = inst->n_machines;
    if (n < 2 || m < 2 || n > PBB_NOALLOC_MAX_N || m > PBB_NOALLOC_MAX_M)
        return na_fail(PBB_E_INVAL,
                       "instance exceeds the no-alloc scratch: at most 64 jobs and 20 machines (2 <= n, 2 <= m)");
    if (johnson_mode < 0 || johnson_mode > 2) return na_fail(PBB_E_UNSUPPORTED, "JohnsonMode must be 0, 1 or 2");
    if (count < 0) return na_fail(PBB_E_INVAL, "count must be >= 0");
    if (count > 0 && (!sched || !limit1 || !limit2 || !weak_begin || !weak_end || !strong_begin || !strong_end ||
                      !node_weak || !node_strong))
        return na_fail(PBB_E_INVAL, "device input and output buffers must all be given");
    if (device < 0 || device >= PBB_NOALLOC_MAX_DEVICES) return na_fail(PBB_E_INVAL, "device index out of range");
    int P = 0, Ppad = 0;
    int rc = na_build_tables(inst, johnson_mode, P, Ppad);
    if (rc != PBB_OK) return rc;
    if (count == 0) return PBB_OK;

    // the caller's current context comes back on every return path below
    pbbh::DeviceGuard keep_callers_device;
    NA_CK(cudaSetDevice(device), "cudaSetDevice failed");
    unsigned char* base = g_scratch_addr[device];
    if (!base) {
        // set-up, once per device, with that device current
        NA_CK(cudaGetSymbolAddress((void**)&base, g_noalloc_scratch), "cudaGetSymbolAddress of the scratch failed");
        NA_CK(cudaDeviceGetAttribute(&g_smem_optin[device], cudaDevAttrMaxSharedMemoryPerBlockOptin, device),
              "device query failed");
        g_scratch_addr[device] = base;
    }
    // block shape: the most warps (up to 8) whose tables and scratch fit the
    // device's per-block shared memory
    int warps = 8, smem = pbbl::smem_bytes(n, m, Ppad, warps);
    while (warps > 1 && smem > g_smem_optin[device]) smem = pbbl::smem_bytes(n, m, Ppad, --warps);
    if (smem > g_smem_optin[device])
        return na_fail(PBB_E_INVAL, "instance tables do not fit in this device's shared memory");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned* status = reinterpret_cast<unsigned*>(base + NA_STATUS_OFF);
    unsigned long long* je = reinterpret_cast<unsigned long long*>(base + NA_JE_OFF);
    int* pd = reinterpret_cast<int*>(base + NA_P_OFF);
    unsigned char* pm = base + NA_PM_OFF;
    int* mt = reinterpret_cast<int*>(base + NA_MT_OFF);
    NA_CK(cudaMemsetAsync(status, 0, sizeof(unsigned), st), "clearing the status word failed");
    NA_CK(cudaMemcpyAsync(je, g_stage.je, sizeof(unsigned long long) * n * Ppad, cudaMemcpyHostToDevice, st),
          "table upload failed");
    NA_CK(cudaMemcpyAsync(pd, g_stage.p, sizeof(int) * n * m, cudaMemcpyHostToDevice, st), "table upload failed");
    NA_CK(cudaMemcpyAsync(pm, g_stage.pm, 2 * Ppad, cudaMemcpyHostToDevice, st), "table upload failed");
    NA_CK(cudaMemcpyAsync(mt, g_stage.mt, sizeof(int) * 2 * m, cudaMemcpyHostToDevice, st), "table upload failed");

    int blocks = (count + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    pbb_noalloc_check_kernel<<<blocks, 256, 0, st>>>(n, count, sched, limit1, limit2);
    NA_CK(cudaGetLastError(), "input check launch failed");
    unsigned hs = 0;
    NA_CK(cudaMemcpyAsync(&hs, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "status read failed");
    NA_CK(cudaStreamSynchronize(st), "input check failed");
    if (hs & PBB_ST_BADINPUT)
        return na_fail(PBB_E_INVAL, "a node is not a permutation of 0..n-1 with -1 <= limit1 < limit2 <= n");

    DevInstance I;
    I.n = n; I.m = m; I.P = P; I.Ppad = Ppad;
    I.p = pd; I.je = je; I.pm0 = pm; I.pm1 = pm + Ppad;
    I.min_arr = mt; I.min_dep = mt + m;
    I.posj = nullptr;   // method 0 (sweeps over all positions) needs no position table
    int sms = 0;
    NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query failed");
    int ctas = (count + warps - 1) / warps;
    if (ctas > sms * 4) ctas = sms * 4;
    NA_CK(pbbl::launch_bound(n <= 32 ? 1 : 2, I, count, sched, limit1, limit2, weak_begin, weak_end, strong_begin,
                             strong_end, node_weak, node_strong, status, ctas, warps, smem, st),
          "bound kernel launch failed");
    NA_CK(cudaMemcpyAsync(&hs, status, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "status read failed");
    NA_CK(cudaStreamSynchronize(st), "bound kernel failed");
    if (hs & PBB_ST_BADINPUT) return na_fail(PBB_E_INVAL, "device rejected a node");
    return PBB_OK;
}
