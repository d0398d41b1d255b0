// Allocation-free variant of the FP64 field tallies (opo_field_sums).
//
// Some callers cannot call cudaMalloc: host frameworks that have reserved the whole
// device memory for their own pool, and loops that cannot afford the implicit
// device-wide synchronisation an allocation may bring.  For them this file keeps the
// reduction's scratch (per-chunk partial sums and the three results) in one
// file-scope device array instead of a buffer allocated per solver.
//
// Capacity: each field is reduced in chunks of kChunk elements, at most kMaxChunks
// chunks, i.e. up to 268,435,456 complex values per field; larger requests are rejected.
// The array (98,328 bytes) is held on every device that loads the library until exit.
// All calls share it, so calls whose work overlaps on the GPU (different streams, or
// different host threads on one device) race and must be ordered by the caller.  Every
// slot a call reads is written earlier in the same call, so nothing needs clearing.

#include "../../include/cuopo3d.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

namespace {

constexpr int kChunk = 65536;
constexpr int kMaxChunks = 4096;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

static __device__ __align__(256) double g_tally_scratch[3 * kMaxChunks + 3];

std::mutex g_setup_mu;
double *g_scratch_addr[kMaxDevices] = {};
thread_local std::string g_noalloc_err;

int report(int code)
{
    fprintf(stderr, "%s\n", g_noalloc_err.c_str());
    return code;
}

// Block b sums chunk b of each field in a fixed order (deterministic).
template <typename C>
__global__ void __launch_bounds__(kThreads) chunk_sums_kernel(const C *f0, const C *f1, const C *f2, size_t n,
                                                              double *scratch)
{
    __shared__ double red[3][kThreads / 32];
    const C *fs[3] = {f0, f1, f2};
    const size_t begin = (size_t)blockIdx.x * kChunk;
    size_t end = begin + kChunk;
    if (end > n) end = n;
    double acc[3] = {0, 0, 0};
    for (size_t v = begin + threadIdx.x; v < end; v += kThreads) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const C a = fs[k][v];
            acc[k] += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double x = acc[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double x = 0;
        for (int w = 0; w < kThreads / 32; w++) x += red[threadIdx.x][w];
        scratch[(size_t)blockIdx.x * 3 + threadIdx.x] = x;
    }
}

__global__ void chunk_total_kernel(double *scratch, int nchunks)
{
    if (threadIdx.x < 3) {
        double x = 0;
        for (int b = 0; b < nchunks; b++) x += scratch[(size_t)b * 3 + threadIdx.x];
        scratch[3 * kMaxChunks + threadIdx.x] = x;
    }
}

// Device address of the scratch array for the current device, looked up once per
// device (the array's name is only a host-side stand-in in host code).
int scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return OPO_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        g_noalloc_err = "device index beyond the supported range";
        return OPO_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_tally_scratch);
        if (e != cudaSuccess || !p) {
            g_noalloc_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return OPO_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return OPO_OK;
}

}  // namespace

extern "C" int opo_field_sums_noalloc(const void *f0, const void *f1, const void *f2, size_t n,
                                      int precision, void *stream, double sums[3])
{
    if (!f0 || !f1 || !f2 || !sums || n == 0 || (precision != OPO_FP32 && precision != OPO_FP64)) {
        g_noalloc_err = "opo_field_sums_noalloc: null pointer, empty field or bad precision";
        return report(OPO_ERR_INVALID);
    }
    const size_t nchunks = (n + kChunk - 1) / kChunk;
    if (nchunks > (size_t)kMaxChunks) {
        g_noalloc_err = "opo_field_sums_noalloc: " + std::to_string(n) +
                        " values per field exceed the fixed capacity of " +
                        std::to_string((size_t)kChunk * kMaxChunks);
        return report(OPO_ERR_CAPACITY);
    }
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return report(rc);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == OPO_FP64)
        chunk_sums_kernel<double2><<<(unsigned)nchunks, kThreads, 0, st>>>(
            (const double2 *)f0, (const double2 *)f1, (const double2 *)f2, n, scratch);
    else
        chunk_sums_kernel<float2><<<(unsigned)nchunks, kThreads, 0, st>>>(
            (const float2 *)f0, (const float2 *)f1, (const float2 *)f2, n, scratch);
    chunk_total_kernel<<<1, 32, 0, st>>>(scratch, (int)nchunks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sums, scratch + 3 * kMaxChunks, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("opo_field_sums_noalloc: ") + cudaGetErrorString(e);
        return report(OPO_ERR_CUDA);
    }
    return OPO_OK;
}
