// FP64 arithmetic peak of the current device, measured: a kernel of independent FMA
// chains (eight per thread, every SM full) timed with CUDA events.  It is the
// denominator of the t-pass's second roofline (the FP64 pipe), next to HBM bandwidth.

#include <cuda_runtime.h>

#include "../../include/cuopo3d.h"

namespace {

constexpr int kChains = 8;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) dfma_chains(const double *seed, double *out, int iters)
{
    const double m = seed[0], c = seed[1];
    double a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; k++) a[k] = seed[2] + k + threadIdx.x * 1e-9;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) a[k] = fma(a[k], m, c);
    }
    double s = 0;
#pragma unroll
    for (int k = 0; k < kChains; k++) s += a[k];
    if (s == 12345.0) out[0] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace

extern "C" int opo_fp64_peak(double *tflops)
{
    if (!tflops) return OPO_ERR_INVALID;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return OPO_ERR_CUDA;
    double *buf = nullptr;
    if (cudaMalloc(&buf, 4 * sizeof(double)) != cudaSuccess) return OPO_ERR_NOMEM;
    const double h[3] = {0.9999999, 1e-9, 1.0};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = OPO_OK;
    do {
        if (cudaMemcpy(buf, h, sizeof(h), cudaMemcpyHostToDevice) != cudaSuccess) { rc = OPO_ERR_CUDA; break; }
        if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) { rc = OPO_ERR_CUDA; break; }
        const int blocks = sms * 8, iters = 1024;
        dfma_chains<<<blocks, kThreads>>>(buf, buf + 3, iters);  // warm-up
        float best = 1e30f;
        for (int r = 0; r < 5; r++) {
            cudaEventRecord(e0);
            dfma_chains<<<blocks, kThreads>>>(buf, buf + 3, iters);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) { rc = OPO_ERR_CUDA; break; }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms;
        }
        if (rc) break;
        const double flops = 2.0 * kChains * (double)iters * blocks * kThreads;
        *tflops = flops / (best * 1e-3) / 1e12;
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    return rc == OPO_OK && cudaGetLastError() != cudaSuccess ? OPO_ERR_CUDA : rc;
}
