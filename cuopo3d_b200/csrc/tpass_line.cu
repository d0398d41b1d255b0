// Kernels of the line-specialised t-pass (tile body in tpass_line.cuh), FP32 and FP64:
//  * tpass_line_kernel: one CTA of 128 threads per tile, four CTAs per SM;
//  * tpass_line_fallback_kernel: the generic tile body at the line variant's CTA size and
//    radix, for grids without a line body.

#include "tpass_line.cuh"

namespace opo {

template <typename C, int NT, int RA, int THREADS>
__global__ void __launch_bounds__(THREADS, 4) tpass_line_kernel(TPassArgs<C> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tpass_line_tile<C, NT, RA, THREADS>(a, blockIdx.x, smem_raw);
}

template <typename C, int R1, int THREADS>
__global__ void __launch_bounds__(THREADS, 4) tpass_line_fallback_kernel(TPassArgs<C> a)
{
    constexpr int RMAX = LineFallback<C, THREADS>::RMAX;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *sm = reinterpret_cast<C *>(smem_raw);
    const C *src[3] = {a.psrc, a.f[1], a.f[2]};
    const unsigned lmask = tpass_load_mask(a);
    for (unsigned tile = blockIdx.x; tile < (unsigned)a.g.ntiles; tile += gridDim.x) {
        stage_tile<C, THREADS, false>(a.g, (unsigned)a.plan.n, tile, src, lmask, sm);
        tpass_tile<C, R1, THREADS, RMAX, true>(a, tile, sm);
    }
}

// Compiled line bodies: (time axis, first-stage radix), CTAs of 128 threads.  Fallback
// radices: FP32 4, 8 and 16, FP64 4.
#define OPO_LINE_SHAPES(X, C) X(C, 256, 16) X(C, 128, 16) X(C, 64, 8)
#define OPO_LINE_ALL(X) OPO_LINE_SHAPES(X, float2) OPO_LINE_SHAPES(X, double2)
#define OPO_LINE_FALLBACKS(X) X(float2, 16) X(float2, 8) X(float2, 4) X(double2, 4)

// A tile and its twiddles (the units are 16 bytes in both precisions; the twiddles are C).
template <typename C> size_t line_smem(int nt, int r1)
{
    if (nt == 256 && r1 == 16) return LineGeom<C, 256, 16>::tile_bytes();
    if (nt == 128 && r1 == 16) return LineGeom<C, 128, 16>::tile_bytes();
    if (nt == 64 && r1 == 8) return LineGeom<C, 64, 8>::tile_bytes();
    return 0;
}
size_t tpass_line_smem(bool fp64, int nt, int r1) { return fp64 ? line_smem<double2>(nt, r1) : line_smem<float2>(nt, r1); }

cudaError_t configure_line_kernels(size_t smem)
{
    cudaError_t e;
#define OPO_SET_L(C, NT, RA)                                                                        \
    if ((e = cudaFuncSetAttribute(tpass_line_kernel<C, NT, RA, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)smem)) != cudaSuccess)                                       \
        return e;
    OPO_LINE_ALL(OPO_SET_L)
#undef OPO_SET_L
#define OPO_SET_F(C, RA)                                                                            \
    if ((e = cudaFuncSetAttribute(tpass_line_fallback_kernel<C, RA, 128>,                           \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;
    OPO_LINE_FALLBACKS(OPO_SET_F)
#undef OPO_SET_F
    return cudaSuccess;
}

template <typename C>
cudaError_t launch_tpass_line(const TPassArgs<C> &a, PassVariant v, int nt, int r_fallback, int grid, size_t smem,
                              cudaStream_t st)
{
    const int r1 = nt ? line_radix(nt) : r_fallback;
    const void *fn = nullptr;
#define OPO_FN_L(CC, NT, RA)                                                                        \
    if constexpr (std::is_same<C, CC>::value)                                                       \
        if (!fn && nt == NT && r1 == RA && v.threads == 128)                                        \
            fn = reinterpret_cast<const void *>(tpass_line_kernel<CC, NT, RA, 128>);
    OPO_LINE_ALL(OPO_FN_L)
#undef OPO_FN_L
#define OPO_FN_F(CC, RA)                                                                            \
    if constexpr (std::is_same<C, CC>::value)                                                       \
        if (!fn && nt == 0 && r1 == RA && v.threads == 128)                                         \
            fn = reinterpret_cast<const void *>(tpass_line_fallback_kernel<CC, RA, 128>);
    OPO_LINE_FALLBACKS(OPO_FN_F)
#undef OPO_FN_F
    if (!fn) return cudaErrorInvalidValue;
    void *args[] = {const_cast<TPassArgs<C> *>(&a)};
    return cudaLaunchKernel(fn, dim3(grid), dim3(v.threads), args, smem, st);
}

template cudaError_t launch_tpass_line<float2>(const TPassArgs<float2> &, PassVariant, int, int, int, size_t,
                                              cudaStream_t);
template cudaError_t launch_tpass_line<double2>(const TPassArgs<double2> &, PassVariant, int, int, int, size_t,
                                               cudaStream_t);

}  // namespace opo
