// Fused (x, y) diffraction pass for sm_100a: one thread-block cluster per (field, t)
// plane, the plane split across the cluster's shared memory.
//
// The diffraction operator of a z-step (Solver3D.cuh:282-323, applied at :954) is the
// product of an x factor and a y factor, each a line transform, a phase multiply and an
// inverse transform.  Run as two passes over HBM (x lines, then y lines) it costs two
// reads and two writes of the fields.  Here a cluster of K CTAs holds a whole plane:
//   1. CTA r loads rows [r ny/K, (r+1) ny/K) of the plane (coalesced row reads), runs the
//      x factor on them in its slab (first forward stage fused with the load, shared-
//      memory middle stages, last inverse stage back into the slab);
//   2. a cluster barrier (release / acquire) publishes every slab to the cluster;
//   3. CTA r gathers columns [r nx/K, (r+1) nx/K) from all K slabs through distributed
//      shared memory, fused with the first forward stage of the y factor, into its
//      column region, arrives on the cluster barrier (its remote reads are done), runs
//      the y factor and writes the columns to global memory from the last inverse stage;
//   4. it waits on the barrier before exiting, so no slab is released while a peer may
//      still read it.
// The fields cross HBM once per z-step for both axes.  The arithmetic (plans, twiddles,
// stage order, tables) is that of the separate x and y passes.

#include <cooperative_groups.h>
#include <type_traits>

#include "pass_body.cuh"

namespace cg = cooperative_groups;

namespace opo {

namespace {

__device__ __forceinline__ void cluster_arrive_release()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire()
{
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Rows of this CTA from global memory, first forward stage (radix R1, sign -1) of the
// x transform, into the slab.  Consecutive threads take consecutive butterflies of a row.
template <typename C, int R1, int THREADS>
__device__ __forceinline__ void load_rows(const PlaneArgs<C> &a, const C *src, C *slab)
{
    const AxisPlan &p = a.px;
    const unsigned n = p.n, q = n / R1, items = q * (unsigned)a.gx.nlines, lsl = a.gx.lsl;
    for (unsigned w = threadIdx.x; w < items; w += THREADS) {
        const unsigned l = fdiv(p.q[0], w), b = w - l * q;
        const C *s = src + l * n + b;
        C x[R1];
#pragma unroll
        for (int m = 0; m < R1; m++) x[m] = s[m * q];
        dft<R1, -1>(x);
#pragma unroll
        for (int k = 1; k < R1; k++) x[k] = twmul<-1>(x[k], __ldg(a.twx + (k - 1) * q + b));
        C *d = slab + l * lsl + b;
#pragma unroll
        for (int k = 0; k < R1; k++) d[k * q] = x[k];
    }
}

// Columns c0 .. c0 + nx/K - 1 gathered from the cluster's slabs (row -> owning CTA),
// first forward stage of the y transform, into the column region (lines contiguous).
template <typename C, int R1, int THREADS>
__device__ __forceinline__ void gather_columns(const PlaneArgs<C> &a, const cg::cluster_group &cl, C *slab,
                                               unsigned c0, C *cols)
{
    const AxisPlan &p = a.py;
    const unsigned n = p.n, q = n / R1, NL = (unsigned)a.gy.nlines, items = q * NL, lsl = a.gx.lsl;
    for (unsigned w = threadIdx.x; w < items; w += THREADS) {
        const unsigned b = fdiv(a.gy.nl, w), l = w - b * NL;
        C x[R1];
#pragma unroll
        for (int m = 0; m < R1; m++) {
            const unsigned row = b + m * q;
            const unsigned owner = fdiv(a.rows, row), lrow = row - owner * a.rows.d;
            const C *peer = cl.map_shared_rank(slab, owner);
            x[m] = peer[lrow * lsl + c0 + l];
        }
        dft<R1, -1>(x);
#pragma unroll
        for (int k = 1; k < R1; k++) x[k] = twmul<-1>(x[k], __ldg(a.twy + (k - 1) * q + b));
        C *d = cols + l + b * NL;
#pragma unroll
        for (int k = 0; k < R1; k++) d[k * q * NL] = x[k];
    }
}

template <typename C, int THREADS, int RMAX>
__device__ __forceinline__ void load_rows_dispatch(const PlaneArgs<C> &a, const C *src, C *slab)
{
    switch (a.px.radix[0]) {
    case 4: load_rows<C, 4, THREADS>(a, src, slab); break;
    case 8: load_rows<C, 8, THREADS>(a, src, slab); break;
    case 16:
        if constexpr (RMAX >= 16) load_rows<C, 16, THREADS>(a, src, slab);
        break;
    default: break;
    }
}

template <typename C, int THREADS, int RMAX>
__device__ __forceinline__ void gather_dispatch(const PlaneArgs<C> &a, const cg::cluster_group &cl, C *slab,
                                                unsigned c0, C *cols)
{
    switch (a.py.radix[0]) {
    case 4: gather_columns<C, 4, THREADS>(a, cl, slab, c0, cols); break;
    case 8: gather_columns<C, 8, THREADS>(a, cl, slab, c0, cols); break;
    case 16:
        if constexpr (RMAX >= 16) gather_columns<C, 16, THREADS>(a, cl, slab, c0, cols);
        break;
    default: break;
    }
}

template <typename C, int THREADS, int RMAX>
__device__ __forceinline__ void store_columns_dispatch(const PlaneArgs<C> &a, C *cols, unsigned base, C *const *dst)
{
    const AxisPlan &p = a.py;
    switch (p.radix[0]) {
    case 4: final_stage<C, 4, +1, false, THREADS>(cols, a.gy, p.n, base, dst, a.twy, p.q[0], 1u); break;
    case 8: final_stage<C, 8, +1, false, THREADS>(cols, a.gy, p.n, base, dst, a.twy, p.q[0], 1u); break;
    case 16:
        if constexpr (RMAX >= 16) final_stage<C, 16, +1, false, THREADS>(cols, a.gy, p.n, base, dst, a.twy, p.q[0], 1u);
        break;
    default: break;
    }
}

}  // namespace

template <typename C, int THREADS, int RMAX>
__global__ void __launch_bounds__(THREADS, THREADS == 256 ? 2 : 1) plane_kernel(PlaneArgs<C> a)
{
    using TT = typename TabOf<C>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *slab = reinterpret_cast<C *>(smem_raw);
    C *cols = slab + a.regionA;
    const cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const unsigned plane = blockIdx.x / a.K;
    const unsigned fsel = plane / a.nt, t = plane - fsel * a.nt;
    const int fid = field_id(a.tmask, (int)fsel);
    C *field = a.f[fid];
    const unsigned pbase = t * a.nx * a.ny;

    // 1. x factor on this CTA's rows
    load_rows_dispatch<C, THREADS, RMAX>(a, field + pbase + rank * a.rows.d * a.nx, slab);
    __syncthreads();
    const TT *tx[1] = {a.tabx[fid]};
    middle_stages<C, -1, THREADS, RMAX>(slab, a.gx, a.px, a.twx, tx, 1u);
    smem_stage_dispatch<C, +1, true, THREADS, RMAX>(a.px.radix[0], slab, a.gx, a.px.n, a.px.len[0], a.px.q[0],
                                                    a.twx + a.px.twoff[0], 1u);
    // 2. every slab of the cluster complete and visible
    cl.sync();
    // 3. y factor on this CTA's columns
    const unsigned c0 = rank * (unsigned)a.gy.nlines;
    gather_dispatch<C, THREADS, RMAX>(a, cl, slab, c0, cols);
    cluster_arrive_release();
    __syncthreads();
    const TT *ty[1] = {a.taby[fid]};
    middle_stages<C, -1, THREADS, RMAX>(cols, a.gy, a.py, a.twy, ty, 1u);
    C *const dst[1] = {field};
    store_columns_dispatch<C, THREADS, RMAX>(a, cols, pbase + c0, dst);
    // 4. peers are done reading this slab
    cluster_wait_acquire();
}

#define OPO_PLANE_VARIANTS(X) X(float2, 256, 16) X(float2, 512, 16) X(double2, 256, 8) X(double2, 512, 8)

cudaError_t configure_plane_kernels(size_t smem)
{
    cudaError_t e;
#define OPO_SET_P(C, T, RM)                                                                         \
    if ((e = cudaFuncSetAttribute(plane_kernel<C, T, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)smem)) != cudaSuccess)                                       \
        return e;
    OPO_PLANE_VARIANTS(OPO_SET_P)
#undef OPO_SET_P
    return cudaSuccess;
}

namespace {

template <typename C> const void *plane_fn(int threads)
{
    const void *fn = nullptr;
#define OPO_FN_P(CC, T, RM)                                                                         \
    if constexpr (std::is_same<C, CC>::value) {                                                     \
        if (!fn && threads == T) fn = reinterpret_cast<const void *>(plane_kernel<CC, T, RM>);      \
    }
    OPO_PLANE_VARIANTS(OPO_FN_P)
#undef OPO_FN_P
    return fn;
}

cudaLaunchConfig_t plane_config(unsigned grid, int threads, int K, size_t smem, cudaStream_t st,
                                cudaLaunchAttribute *attr)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3((unsigned)threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

}  // namespace

template <typename C>
cudaError_t launch_plane(const PlaneArgs<C> &a, int threads, unsigned planes, size_t smem, cudaStream_t st)
{
    const void *fn = plane_fn<C>(threads);
    if (!fn || a.K < 2 || a.K > 8) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_config(planes * a.K, threads, (int)a.K, smem, st, attr);
    void *args[1] = {const_cast<PlaneArgs<C> *>(&a)};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

template <typename C> int plane_max_clusters(int threads, int K, size_t smem)
{
    const void *fn = plane_fn<C>(threads);
    if (!fn || K < 2 || K > 8) return 0;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = plane_config((unsigned)K, threads, K, smem, nullptr, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n;
}

template cudaError_t launch_plane<float2>(const PlaneArgs<float2> &, int, unsigned, size_t, cudaStream_t);
template cudaError_t launch_plane<double2>(const PlaneArgs<double2> &, int, unsigned, size_t, cudaStream_t);
template int plane_max_clusters<float2>(int, int, size_t);
template int plane_max_clusters<double2>(int, int, size_t);

}  // namespace opo
