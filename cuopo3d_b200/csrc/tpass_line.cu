// Single-instance kernels of the line-specialised FP32 t-pass (tile body in
// tpass_line.cuh): one CTA per tile of 8 pixels x NT samples x 3 fields.

#include "tpass_line.cuh"

namespace opo {

template <int NT, int RA, int THREADS>
__global__ void __launch_bounds__(THREADS, 4) tpass_line_kernel(TPassArgs<float2> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tpass_line_tile<NT, RA, THREADS>(a, blockIdx.x, reinterpret_cast<float2 *>(smem_raw));
}

// Grids without a line body: the generic FP32 tile body at the same CTA size and
// first-stage radix (the body the batched kernel runs for such instances).
template <int R1, int THREADS>
__global__ void __launch_bounds__(THREADS, 4) tpass_line_fallback_kernel(TPassArgs<float2> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *sm = reinterpret_cast<float2 *>(smem_raw);
    const float2 *src[3] = {a.psrc, a.f[1], a.f[2]};
    const unsigned lmask = tpass_load_mask(a);
    for (unsigned tile = blockIdx.x; tile < (unsigned)a.g.ntiles; tile += gridDim.x) {
        stage_tile<float2, THREADS, false>(a.g, (unsigned)a.plan.n, tile, src, lmask, sm);
        tpass_tile<float2, R1, THREADS, 16, true>(a, tile, sm);
    }
}

// Compiled (time axis, first-stage radix) shapes x CTA sizes; CTA sizes x radices of the
// fallback.
#define OPO_LINE_VARIANTS(X)                                                                       \
    X(256, 16, 128) X(128, 16, 128) X(64, 8, 128) X(256, 16, 96) X(128, 16, 96) X(64, 8, 96)
#define OPO_LINE_FALLBACKS(X) X(16, 128) X(8, 128) X(16, 96) X(8, 96)

size_t tpass_line_smem(int nt, int r1)
{
    if (nt == 256 && r1 == 16) return LineGeom<256, 16>::smem_bytes();
    if (nt == 128 && r1 == 16) return LineGeom<128, 16>::smem_bytes();
    if (nt == 64 && r1 == 8) return LineGeom<64, 8>::smem_bytes();
    return 0;
}

cudaError_t configure_line_kernels(size_t smem)
{
    cudaError_t e;
#define OPO_SET_L(NT, RA, T)                                                                        \
    if ((e = cudaFuncSetAttribute(tpass_line_kernel<NT, RA, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)smem)) != cudaSuccess)                                       \
        return e;
    OPO_LINE_VARIANTS(OPO_SET_L)
#undef OPO_SET_L
#define OPO_SET_F(RA, T)                                                                            \
    if ((e = cudaFuncSetAttribute(tpass_line_fallback_kernel<RA, T>,                                \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;
    OPO_LINE_FALLBACKS(OPO_SET_F)
#undef OPO_SET_F
    return cudaSuccess;
}

cudaError_t launch_tpass_line(const TPassArgs<float2> &a, PassVariant v, int nt, int grid, size_t smem,
                              cudaStream_t st)
{
    const int r1 = radix_of(v);
    bool done = false;
#define OPO_LAUNCH_L(NT, RA, T)                                                                     \
    if (!done && nt == NT && r1 == RA && v.threads == T) {                                          \
        tpass_line_kernel<NT, RA, T><<<grid, T, smem, st>>>(a);                                     \
        done = true;                                                                                \
    }
    OPO_LINE_VARIANTS(OPO_LAUNCH_L)
#undef OPO_LAUNCH_L
#define OPO_LAUNCH_F(RA, T)                                                                         \
    if (!done && r1 == RA && v.threads == T) {                                                      \
        tpass_line_fallback_kernel<RA, T><<<grid, T, smem, st>>>(a);                                \
        done = true;                                                                                \
    }
    OPO_LINE_FALLBACKS(OPO_LAUNCH_F)
#undef OPO_LAUNCH_F
    return done ? cudaGetLastError() : cudaErrorInvalidValue;
}

}  // namespace opo
