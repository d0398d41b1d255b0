// Allocation-free variant of the FP64 field tallies (opo_field_sums).
//
// Some callers cannot call cudaMalloc: host frameworks that have reserved the whole
// device memory for their own pool, and loops that cannot afford the implicit
// device-wide synchronisation an allocation may bring.  For them this file keeps the
// reduction's scratch (per-block partial sums and the three results) in one
// file-scope device array instead of a buffer allocated per solver.
//
// Capacity: up to 268,435,456 complex values per field; larger requests are rejected.
// The fields are cut into chunks of kChunk values; a grid of min(chunks, kMaxBlocks)
// blocks takes chunk b, b + grid, b + 2 grid, ... per block in that order, so the
// summation order, and with it the result, depends only on n.  The array (24,600
// bytes) is held on every device that loads the library until exit.  All calls share
// it, so calls whose work overlaps on the GPU (different streams, or different host
// threads on one device) race and must be ordered by the caller.  Every slot a call
// reads is written earlier in the same call, so nothing needs clearing.

#include "../../include/cuopo3d.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

namespace {

constexpr int kChunk = 8192;
constexpr int kMaxBlocks = 1024;
constexpr size_t kMaxValues = (size_t)1 << 28;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

static __device__ __align__(256) double g_tally_scratch[3 * kMaxBlocks + 3];

std::mutex g_setup_mu;
// per device: the scratch array's device address and the id of the CUDA context it was
// looked up in (a context made after cudaDeviceReset may place the array elsewhere)
double *g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};
thread_local std::string g_noalloc_err;

// Block b sums chunks b, b + gridDim.x, ... of each field, in that order (deterministic
// for a given n), and writes its three partial sums.
template <typename C>
__global__ void __launch_bounds__(kThreads) chunk_sums_kernel(const C *f0, const C *f1, const C *f2, size_t n,
                                                              double *scratch)
{
    __shared__ double red[3][kThreads / 32];
    const C *fs[3] = {f0, f1, f2};
    const size_t nchunks = (n + kChunk - 1) / kChunk;
    double acc[3] = {0, 0, 0};
    for (size_t c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const size_t begin = c * kChunk;
        const size_t end = begin + kChunk < n ? begin + kChunk : n;
        for (size_t v = begin + threadIdx.x; v < end; v += kThreads) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const C a = fs[k][v];
                acc[k] += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
            }
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

__global__ void chunk_total_kernel(double *scratch, int nblocks)
{
    if (threadIdx.x < 3) {
        double x = 0;
        for (int b = 0; b < nblocks; b++) x += scratch[(size_t)b * 3 + threadIdx.x];
        scratch[3 * kMaxBlocks + threadIdx.x] = x;
    }
}

// Id of the current CUDA context (cuCtxGetCurrent + cuCtxGetId through the runtime's
// driver entry points, so the library needs no link to libcuda); 0 if unavailable.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
        (void)cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array for the current device, looked up once per device
// and context (the array's name is only a host-side stand-in in host code).
int scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("opo_field_sums_noalloc: cudaGetDevice: ") + cudaGetErrorString(e);
        return OPO_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        g_noalloc_err = "opo_field_sums_noalloc: device index beyond the supported range";
        return OPO_ERR_INVALID;
    }
    // id 0: no context yet (the symbol lookup creates it) or the id is not available, in
    // which case the address is looked up on every call
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev] || ctx == 0 || ctx != g_scratch_ctx[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_tally_scratch);
        if (e != cudaSuccess || !p) {
            g_noalloc_err = std::string("opo_field_sums_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return OPO_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
        g_scratch_ctx[dev] = current_context_id();
    }
    *out = g_scratch_addr[dev];
    return OPO_OK;
}

}  // namespace

extern "C" const char *opo_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" int opo_field_sums_noalloc(const void *f0, const void *f1, const void *f2, size_t n,
                                      int precision, void *stream, double sums[3])
{
    g_noalloc_err.clear();
    if (!f0 || !f1 || !f2 || !sums || n == 0 || (precision != OPO_FP32 && precision != OPO_FP64)) {
        g_noalloc_err = "opo_field_sums_noalloc: null pointer, empty field or bad precision";
        return OPO_ERR_INVALID;
    }
    if (n > kMaxValues) {
        g_noalloc_err = "opo_field_sums_noalloc: " + std::to_string(n) +
                        " values per field exceed the fixed capacity of " + std::to_string(kMaxValues);
        return OPO_ERR_CAPACITY;
    }
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    const size_t nchunks = (n + kChunk - 1) / kChunk;
    const unsigned nblocks = (unsigned)(nchunks < (size_t)kMaxBlocks ? nchunks : (size_t)kMaxBlocks);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == OPO_FP64)
        chunk_sums_kernel<double2><<<nblocks, kThreads, 0, st>>>((const double2 *)f0, (const double2 *)f1,
                                                                 (const double2 *)f2, n, scratch);
    else
        chunk_sums_kernel<float2><<<nblocks, kThreads, 0, st>>>((const float2 *)f0, (const float2 *)f1,
                                                                (const float2 *)f2, n, scratch);
    chunk_total_kernel<<<1, 32, 0, st>>>(scratch, (int)nblocks);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sums, scratch + 3 * kMaxBlocks, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        g_noalloc_err = std::string("opo_field_sums_noalloc: ") + cudaGetErrorString(e);
        return OPO_ERR_CUDA;
    }
    if (!std::isfinite(sums[0]) || !std::isfinite(sums[1]) || !std::isfinite(sums[2])) {
        g_noalloc_err = "opo_field_sums_noalloc: the fields hold non-finite values";
        return OPO_ERR_NONFINITE;
    }
    return OPO_OK;
}
