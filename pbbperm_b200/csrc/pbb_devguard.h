// Entry points select their device with cudaSetDevice.  A library called from
// inside another framework (torch, a plugin host) must not leave a different
// device current for its caller: DeviceGuard saves the calling thread's
// current CUDA context on entry and puts it back on every return path.  The
// driver's context calls are reached through cudaGetDriverEntryPoint, so the
// library still loads on machines without a driver (no link against libcuda).
#pragma once
#include <cuda_runtime.h>

namespace pbbh {

struct CtxApi {
    int (*get)(void**) = nullptr;   // cuCtxGetCurrent
    int (*set)(void*) = nullptr;    // cuCtxSetCurrent
};

inline const CtxApi& ctx_api()
{
    static const CtxApi api = [] {
        CtxApi a;
        void* g = nullptr;
        void* s = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &g, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxSetCurrent", &s, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess && g && s) {
            a.get = reinterpret_cast<int (*)(void**)>(g);
            a.set = reinterpret_cast<int (*)(void*)>(s);
        }
        cudaGetLastError();   // a failed lookup must not surface as a later error
        return a;
    }();
    return api;
}

class DeviceGuard {
public:
    DeviceGuard()
    {
        const CtxApi& a = ctx_api();
        if (a.get && a.get(&ctx_) == 0) saved_ = true;
    }
    ~DeviceGuard()
    {
        // a thread that had no current context gets none back (restoring
        // "device 0" would create a context there)
        if (saved_) ctx_api().set(ctx_);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

private:
    void* ctx_ = nullptr;
    bool saved_ = false;
};

}  // namespace pbbh
