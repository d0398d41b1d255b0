// Single-instance pass kernels of the split-step solver for sm_100a (the tile bodies
// are in pass_body.cuh), the FP64 tallies, precision conversions and the launchers.

#include <type_traits>

#include "pass_body.cuh"

namespace opo {

// Single-instance kernels: the grid walks the tiles of one solver.  Several CTAs per SM
// (each a tile of 3 fields in shared memory) overlap one another's global loads, the
// shared-memory stages and the stores.  The t-pass stages its whole tile with cp.async
// first (one memory latency per tile for its 12 loads per item); the axis passes, with
// fewer values per item, load straight into registers in their first stage, which
// measured faster for them.

template <typename C, int R1, int THREADS, int RMAX>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 4 : 1) tpass_kernel(TPassArgs<C> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    const C *src[3] = {a.psrc, a.f[1], a.f[2]};
    const unsigned lmask = tpass_load_mask(a);
    for (unsigned tile = blockIdx.x; tile < (unsigned)a.g.ntiles; tile += gridDim.x) {
        stage_tile<C, THREADS, false>(a.g, (unsigned)a.plan.n, tile, src, lmask, sm);
        tpass_tile<C, R1, THREADS, RMAX, true>(a, tile, sm);
    }
}

template <typename C, int R1, bool BFAST, int THREADS, int RMAX>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 4 : 1) axis_kernel(AxisArgs<C> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    for (unsigned tile = blockIdx.x; tile < (unsigned)a.g.ntiles; tile += gridDim.x)
        axis_tile<C, R1, BFAST, THREADS, RMAX>(a, tile, sm);
}

// ---------------------------------------------------------------------------------
// FP64 sums of |A|^2 for three fields: per-block partials, then one block adds the
// partials in a fixed order (deterministic).

constexpr int kSumThreads = 256;

template <typename C>
__global__ void __launch_bounds__(kSumThreads) sums_partial_kernel(const C *f0, const C *f1, const C *f2,
                                                                    size_t n, double *partials)
{
    __shared__ double red[3][kSumThreads / 32];
    double acc[3] = {0, 0, 0};
    const C *fs[3] = {f0, f1, f2};
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            C a = fs[k][v];
            acc[k] += (double)a.x * (double)a.x + (double)a.y * (double)a.y;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 0;
        for (int wv = 0; wv < kSumThreads / 32; wv++) v += red[threadIdx.x][wv];
        partials[(size_t)blockIdx.x * 3 + threadIdx.x] = v;
    }
}

__global__ void sums_final_kernel(const double *partials, int nblocks, double *out)
{
    if (threadIdx.x < 3) {
        double v = 0;
        for (int b = 0; b < nblocks; b++) v += partials[(size_t)b * 3 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

__global__ void convert_d2f_kernel(const double2 *src, float2 *dst, size_t n)
{
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x)
        dst[v] = make_float2((float)src[v].x, (float)src[v].y);
}

__global__ void convert_f2d_kernel(const float2 *src, double2 *dst, size_t n)
{
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (size_t)gridDim.x * blockDim.x)
        dst[v] = make_double2(src[v].x, src[v].y);
}

// ---------------------------------------------------------------------------------
// Compiled variants: (element type, threads, first-stage radix, largest radix).

#define OPO_T_VARIANTS(X)                                                                          \
    X(float2, 128, 4, 16) X(float2, 128, 8, 16) X(float2, 128, 16, 16) X(float2, 256, 4, 16)        \
    X(float2, 256, 8, 16) X(float2, 256, 16, 16) X(double2, 128, 4, 8) X(double2, 128, 8, 8)        \
    X(double2, 256, 4, 16) X(double2, 256, 8, 16)

#define OPO_A_VARIANTS(X)                                                                          \
    X(float2, 128, 4, 16) X(float2, 128, 8, 16) X(float2, 128, 16, 16) X(float2, 256, 4, 16)        \
    X(float2, 256, 8, 16) X(float2, 256, 16, 16) X(double2, 128, 4, 8) X(double2, 128, 8, 8)        \
    X(double2, 256, 4, 16) X(double2, 256, 8, 16) X(double2, 256, 16, 16)

cudaError_t configure_kernels(size_t smem)
{
    cudaError_t e;
#define OPO_SET_T(C, T, R, RM)                                                                      \
    if ((e = cudaFuncSetAttribute(tpass_kernel<C, R, T, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)smem)) != cudaSuccess)                                       \
        return e;
#define OPO_SET_A(C, T, R, RM)                                                                      \
    if ((e = cudaFuncSetAttribute(axis_kernel<C, R, true, T, RM>,                                   \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;                                                                                   \
    if ((e = cudaFuncSetAttribute(axis_kernel<C, R, false, T, RM>,                                  \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;
    OPO_T_VARIANTS(OPO_SET_T)
    OPO_A_VARIANTS(OPO_SET_A)
#undef OPO_SET_T
#undef OPO_SET_A
    return cudaSuccess;
}

template <typename C>
cudaError_t launch_tpass(const TPassArgs<C> &a, PassVariant v, int grid, size_t smem, cudaStream_t st)
{
    bool done = false;
#define OPO_LAUNCH_T(CC, T, R, RM)                                                                  \
    if constexpr (std::is_same<C, CC>::value) {                                                     \
        if (!done && v.threads == T && v.r1 == R) {                                                 \
            tpass_kernel<CC, R, T, RM><<<grid, T, smem, st>>>(a);                                   \
            done = true;                                                                            \
        }                                                                                           \
    }
    OPO_T_VARIANTS(OPO_LAUNCH_T)
#undef OPO_LAUNCH_T
    return done ? cudaGetLastError() : cudaErrorInvalidValue;
}

template <typename C>
cudaError_t launch_axis(const AxisArgs<C> &a, PassVariant v, bool bfast, int grid, size_t smem, cudaStream_t st)
{
    bool done = false;
#define OPO_LAUNCH_A(CC, T, R, RM)                                                                  \
    if constexpr (std::is_same<C, CC>::value) {                                                     \
        if (!done && v.threads == T && v.r1 == R) {                                                 \
            if (bfast) axis_kernel<CC, R, true, T, RM><<<grid, T, smem, st>>>(a);                   \
            else axis_kernel<CC, R, false, T, RM><<<grid, T, smem, st>>>(a);                        \
            done = true;                                                                            \
        }                                                                                           \
    }
    OPO_A_VARIANTS(OPO_LAUNCH_A)
#undef OPO_LAUNCH_A
    return done ? cudaGetLastError() : cudaErrorInvalidValue;
}

template <typename C>
cudaError_t launch_sums(const C *f0, const C *f1, const C *f2, size_t n, double *partials, int nblocks,
                        double *out, cudaStream_t st)
{
    sums_partial_kernel<C><<<nblocks, kSumThreads, 0, st>>>(f0, f1, f2, n, partials);
    sums_final_kernel<<<1, 32, 0, st>>>(partials, nblocks, out);
    return cudaGetLastError();
}

cudaError_t launch_convert_d2f(const double2 *src, float2 *dst, size_t n, cudaStream_t st)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    convert_d2f_kernel<<<blocks, 256, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_convert_f2d(const float2 *src, double2 *dst, size_t n, cudaStream_t st)
{
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    convert_f2d_kernel<<<blocks, 256, 0, st>>>(src, dst, n);
    return cudaGetLastError();
}

template cudaError_t launch_tpass<float2>(const TPassArgs<float2> &, PassVariant, int, size_t, cudaStream_t);
template cudaError_t launch_tpass<double2>(const TPassArgs<double2> &, PassVariant, int, size_t, cudaStream_t);
template cudaError_t launch_axis<float2>(const AxisArgs<float2> &, PassVariant, bool, int, size_t, cudaStream_t);
template cudaError_t launch_axis<double2>(const AxisArgs<double2> &, PassVariant, bool, int, size_t, cudaStream_t);
template cudaError_t launch_sums<float2>(const float2 *, const float2 *, const float2 *, size_t, double *, int,
                                         double *, cudaStream_t);
template cudaError_t launch_sums<double2>(const double2 *, const double2 *, const double2 *, size_t, double *,
                                          int, double *, cudaStream_t);

}  // namespace opo
