// Diagnostic: measured INT32 throughput of this GPU (the denominator of the
// engine's roofline -- its bound kernels are integer add/max issue bound).
//
// Each thread runs 8 independent chains of  a = max(a + x, y)  (one IADD and
// one IMNMX per step), so the loop has no dependency stalls once 4+ warps per
// scheduler are resident.  Ops counted = 2 per step per chain.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "../../include/pbbperm_diag.h"
#include "pbb_devguard.h"

#define DIAG_CHAINS 8

__global__ void pbb_diag_int32_kernel(int iters, int seed, int* out)
{
    int a[DIAG_CHAINS], x[DIAG_CHAINS], y[DIAG_CHAINS];
#pragma unroll
    for (int c = 0; c < DIAG_CHAINS; c++) {
        a[c] = threadIdx.x + c * seed;
        x[c] = (seed * (c + 1)) % 17 - 8;
        y[c] = (int)blockIdx.x - c;
    }
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
#pragma unroll
            for (int c = 0; c < DIAG_CHAINS; c++) a[c] = max(a[c] + x[c], y[c]);
        }
    }
    int s = 0;
#pragma unroll
    for (int c = 0; c < DIAG_CHAINS; c++) s ^= a[c];
    if (s == 0x7fffffff) out[0] = s;   // never true in practice; keeps the chains live
}

extern "C" int pbb_diag_int32_peak(int32_t device, double* gops, double* seconds)
{
    if (!gops) return -1;
    pbbh::DeviceGuard keep_callers_device;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int* out = nullptr;
    if (cudaMalloc(&out, sizeof(int)) != cudaSuccess) return -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int threads = 1024, blocks = sms * 2, iters = 4096;
    pbb_diag_int32_kernel<<<blocks, threads>>>(64, 3, out);   // warm-up
    cudaEventRecord(e0);
    pbb_diag_int32_kernel<<<blocks, threads>>>(iters, 3, out);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return -3;
    const double ops = 2.0 * DIAG_CHAINS * 16.0 * iters * (double)threads * blocks;
    *gops = ops / (ms * 1e-3) / 1e9;
    if (seconds) *seconds = ms * 1e-3;
    return 0;
}
