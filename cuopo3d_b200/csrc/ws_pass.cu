// Warp-specialised persistent pass kernels for sm_100a.
//
// A CTA is NC consumer threads (NC/32 warps) plus one producer warp.  The producer
// streams the CTA's tiles into a ring of shared-memory stages with the Tensor Memory
// Accelerator: t and y tiles as tensor copies (cp.async.bulk.tensor over the field
// viewed as a 3-D tensor (nx, ny, nt) of 8-byte elements, one box per field and up to
// 256 lines), x tiles as one bulk copy (cp.async.bulk) per row.  Each stage has a "full"
// mbarrier (the producer's expect_tx, completed by the copies' byte count) and an
// "empty" mbarrier (one arrival per consumer warp when the tile is done).  Consumers run
// the same tile bodies as the other kernels (first stage from the staged tile, shared-
// memory middle stages, last inverse stage straight to global memory), synchronising
// among themselves with named barrier 1 -- never with the producer -- so the loads of
// the next tiles are in flight while a tile is computed, and no register holds data in
// flight.
//
// Every mbarrier wait is bounded (iteration count and clock): on expiry the waiting side
// records an error code in global memory and leaves its loop; the consumers agree on
// leaving through a shared flag read after a consumer barrier, and the producer drains
// (with a bounded wait) the copies it issued before the CTA exits.  The host reads the
// error word when it next synchronises with the solver.
//
// No copy uses cluster multicast; the kernels are launched without clusters.

#include <type_traits>

#include "pass_body.cuh"

namespace opo {

namespace {

constexpr long long kWaitCycles = 4000000000ll;  // ~2 s at 2 GHz
constexpr unsigned kWaitIters = 1u << 28;

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the completion of the phase of parity `parity`; false when the bound
// (`cycles` SM clock cycles, or kWaitIters polls) expires.  try_wait may suspend the
// thread until the phase completes within a hardware time window, so a bound shorter
// than the default polls with the non-blocking test_wait instead: then the bound, not
// that window, ends the wait.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, long long cycles = kWaitCycles)
{
    const long long t0 = clock64();
    if (cycles < kWaitCycles) {
        for (unsigned it = 0; it < kWaitIters; it++) {
            if (mbar_test_wait(bar, parity)) return true;
            if (clock64() - t0 > cycles) break;
        }
        return false;
    }
    for (unsigned it = 0; it < kWaitIters; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > cycles) break;
    }
    return false;
}
__device__ __forceinline__ long long ring_wait_cycles(const WsArgs &w) { return w.wait_cycles > 0 ? w.wait_cycles : kWaitCycles; }

__device__ __forceinline__ void tma_tensor_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                              unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_bulk(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Orders the consumers' generic-proxy accesses to a stage before the next tensor / bulk
// copy into it.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

template <typename C> __device__ __forceinline__ C *stage_ptr(unsigned char *base, const WsArgs &w, unsigned s)
{
    return reinterpret_cast<C *>(base + (size_t)s * w.stage_bytes);
}

// Issue the copies of tile `tile` (fields in mask) into stage memory `sm`; the lanes of
// the producer warp split them.  Completion is counted on `bar`.
template <typename C>
__device__ __forceinline__ void issue_tile(const WsArgs &w, const TileGeom &g, unsigned tile, unsigned mask,
                                           const CUtensorMap *const *maps, C *const *rowsrc, C *sm,
                                           unsigned long long *bar, unsigned lane)
{
    const unsigned hi = fdiv(g.tdiv, tile), lo = tile - hi * g.tdiv.d;
    unsigned k = 0;
    if (w.mode == kWsTensor) {
        const int c0 = (int)(lo * w.px * w.inner_mult);
        const unsigned chunks = w.lines / w.box_lines;
        for (int f = 0; f < 3; f++) {
            if (!(mask & (1u << f))) continue;
            for (unsigned c = 0; c < chunks; c++, k++) {
                if ((k & 31u) != lane) continue;
                const int line0 = (int)(c * w.box_lines);
                C *dst = sm + (size_t)f * g.region + (size_t)line0 * g.lsj;
                if (w.line_dim == 2)
                    tma_tensor_3d(dst, maps[f], c0, (int)hi, line0, bar);  // t-pass: (x block, row y, t lines)
                else
                    tma_tensor_3d(dst, maps[f], c0, line0, (int)hi, bar);  // y-pass: (x block, y lines, plane t)
            }
        }
    } else {
        // x tile: g.nlines rows, contiguous in global memory, row stride g.lsl in shared memory
        const unsigned base = lo * g.tmulA + hi * g.tmulB;
        const unsigned rows = (unsigned)g.nlines;
        for (int f = 0; f < 3; f++) {
            if (!(mask & (1u << f))) continue;
            for (unsigned l = 0; l < rows; l++, k++)
                if ((k & 31u) == lane)
                    tma_bulk(sm + (size_t)f * g.region + l * g.lsl, rowsrc[f] + base + l * g.gs_l, w.row_bytes, bar);
        }
    }
}

// Producer warp: fill stage k % nstages with tile k once the consumers released it.
template <typename C>
__device__ __forceinline__ void producer_loop(const WsArgs &w, const TileGeom &g, unsigned mask,
                                              const CUtensorMap *const *maps, C *const *rowsrc, unsigned char *stages,
                                              unsigned long long *full, unsigned long long *empty)
{
    const unsigned lane = threadIdx.x & 31u;
    const unsigned ntiles = (unsigned)g.ntiles, nst = w.nstages;
    const unsigned tile_bytes = (unsigned)__popc(mask) * w.field_bytes;
    unsigned k = 0;
    for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
        const unsigned s = k % nst, use = k / nst;
        if (use > 0) {
            int got = 1;
            if (lane == 0) got = mbar_wait(&empty[s], (use - 1) & 1u, ring_wait_cycles(w)) ? 1 : 0;
            got = __shfl_sync(0xffffffffu, got, 0);
            if (!got) {
                if (lane == 0) atomicExch(w.err, 1);
                break;
            }
        }
        if (lane == 0) mbar_arrive_expect_tx(&full[s], tile_bytes);
        __syncwarp();
        issue_tile<C>(w, g, tile, mask, maps, rowsrc, stage_ptr<C>(stages, w, s), &full[s], lane);
    }
    // drain: every issued copy has landed before the CTA may exit (its stages go away);
    // this wait keeps the full bound whatever ring_wait_cycles is: the copies are issued
    // and complete within microseconds.  Should it still expire (code 2), copies may land
    // after the CTA exited, so the host treats every nonzero code as fields lost.
    if (lane == 0)
        for (unsigned j = k > nst ? k - nst : 0; j < k; j++)
            if (!mbar_wait(&full[j % nst], (j / nst) & 1u)) {
                atomicExch(w.err, 2);
                break;
            }
}

// Consumer warps: wait for the stage, agree on leaving after a failed wait, run the body
// (which ends with a consumer barrier), release the stage.
template <int NC, typename Body>
__device__ __forceinline__ void consumer_loop(const WsArgs &w, unsigned ntiles, unsigned long long *full,
                                              unsigned long long *empty, volatile int *abort_flag, Body body)
{
    unsigned k = 0;
    for (unsigned tile = blockIdx.x; tile < ntiles; tile += gridDim.x, k++) {
        const unsigned s = k % w.nstages, use = k / w.nstages;
        if (!mbar_wait(&full[s], use & 1u, ring_wait_cycles(w))) {
            *abort_flag = 1;
            atomicExch(w.err, 3);
        }
        tile_sync<NC>();
        if (*abort_flag) return;
        body(tile, s);
        fence_proxy_async_smem();
        __syncwarp();
        if ((threadIdx.x & 31u) == 0) mbar_arrive(&empty[s]);
    }
}

__device__ __forceinline__ void init_ring(const WsArgs &w, unsigned long long *full, unsigned long long *empty,
                                          volatile int *abort_flag, unsigned consumer_warps)
{
    if (threadIdx.x == 0) {
        for (unsigned s = 0; s < w.nstages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], consumer_warps);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
}

}  // namespace

// ---------------------------------------------------------------------------------

template <typename C, int R1, int NC, int RMAX>
__global__ void __launch_bounds__(NC + 32, NC == 128 ? 2 : 1)
    tpass_ws_kernel(TPassArgs<C> a, WsArgs w, const __grid_constant__ CUtensorMap m0,
                    const __grid_constant__ CUtensorMap m1, const __grid_constant__ CUtensorMap m2)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned long long *full = reinterpret_cast<unsigned long long *>(smem_raw);
    unsigned long long *empty = full + kWsMaxStages;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + kWsMaxStages);
    unsigned char *stages = smem_raw + kWsHeaderBytes;
    init_ring(w, full, empty, abort_flag, NC / 32);
    if (threadIdx.x >= NC) {
        const CUtensorMap *maps[3] = {&m0, &m1, &m2};
        C *rows[3] = {nullptr, nullptr, nullptr};
        producer_loop<C>(w, a.g, tpass_load_mask(a), maps, rows, stages, full, empty);
        return;
    }
    consumer_loop<NC>(w, (unsigned)a.g.ntiles, full, empty, abort_flag, [&](unsigned tile, unsigned s) {
        tpass_tile<C, R1, NC, RMAX, true, NC>(a, tile, stage_ptr<C>(stages, w, s));
    });
}

template <typename C, int R1, bool BFAST, int NC, int RMAX>
__global__ void __launch_bounds__(NC + 32, NC == 128 ? 2 : 1)
    axis_ws_kernel(AxisArgs<C> a, WsArgs w, const __grid_constant__ CUtensorMap m0,
                   const __grid_constant__ CUtensorMap m1, const __grid_constant__ CUtensorMap m2)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned long long *full = reinterpret_cast<unsigned long long *>(smem_raw);
    unsigned long long *empty = full + kWsMaxStages;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + kWsMaxStages);
    unsigned char *stages = smem_raw + kWsHeaderBytes;
    if (!a.tmask) return;
    init_ring(w, full, empty, abort_flag, NC / 32);
    if (threadIdx.x >= NC) {
        const CUtensorMap *maps[3] = {&m0, &m1, &m2};
        producer_loop<C>(w, a.g, a.tmask, maps, a.f, stages, full, empty);
        return;
    }
    using TT = typename TabOf<C>::type;
    const C *tw = a.tw;
    const TT *const *tab = a.tab;
    if (w.tab_off) {
        // the pass's stage twiddles and phase tables, read by every tile, into shared
        // memory; the three table pointers sit in the header (indexed by field at run time)
        C *tws = reinterpret_cast<C *>(smem_raw + w.tab_off);
        for (unsigned i = threadIdx.x; i < w.ntw; i += NC) tws[i] = a.tw[i];
        TT *tb = reinterpret_cast<TT *>(tws + w.ntw);
        const TT **tabs = reinterpret_cast<const TT **>(smem_raw + kWsTabPtrOffset);
        const unsigned n = (unsigned)a.plan.n;
        for (int f = 0; f < 3; f++) {
            if (!(a.tmask & (1u << f))) continue;
            for (unsigned i = threadIdx.x; i < n; i += NC) tb[i] = a.tab[f][i];
            if (threadIdx.x == 0) tabs[f] = tb;
            tb += n;
        }
        tile_sync<NC>();
        tw = tws;
        tab = tabs;
    }
    consumer_loop<NC>(w, (unsigned)a.g.ntiles, full, empty, abort_flag, [&](unsigned tile, unsigned s) {
        axis_tile<C, R1, BFAST, NC, RMAX, true, NC>(a, tile, stage_ptr<C>(stages, w, s), tw, tab);
    });
}

// ---------------------------------------------------------------------------------
// Compiled variants (element type, consumer threads, first-stage radix, largest radix).
// Consumer warps have 168-204 registers, so every variant allows radix-16 stages.

#define OPO_WS_T_VARIANTS(X)                                                                        \
    X(float2, 128, 4, 16) X(float2, 256, 4, 16) X(float2, 256, 8, 16) X(double2, 128, 4, 16)         \
    X(double2, 256, 4, 16) X(double2, 256, 8, 16)
#define OPO_WS_A_VARIANTS(X)                                                                        \
    X(float2, 128, 8, 16) X(float2, 128, 16, 16) X(float2, 256, 16, 16) X(double2, 128, 4, 16)       \
    X(double2, 128, 8, 16) X(double2, 256, 8, 16)

cudaError_t configure_ws_kernels(size_t smem)
{
    cudaError_t e;
#define OPO_SET_WT(C, T, R, RM)                                                                     \
    if ((e = cudaFuncSetAttribute(tpass_ws_kernel<C, R, T, RM>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)smem)) != cudaSuccess)                                       \
        return e;
#define OPO_SET_WA(C, T, R, RM)                                                                     \
    if ((e = cudaFuncSetAttribute(axis_ws_kernel<C, R, true, T, RM>,                                \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;                                                                                   \
    if ((e = cudaFuncSetAttribute(axis_ws_kernel<C, R, false, T, RM>,                               \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess) \
        return e;
    OPO_WS_T_VARIANTS(OPO_SET_WT)
    OPO_WS_A_VARIANTS(OPO_SET_WA)
#undef OPO_SET_WT
#undef OPO_SET_WA
    return cudaSuccess;
}

bool ws_variant_compiled(bool fp64, bool tpass, PassVariant v)
{
    bool ok = false;
    const int T = v.threads, R = v.r1;
#define OPO_HAS_WT(CC, TT, RR, RM)                                                                  \
    if (tpass && (sizeof(CC) == 16) == fp64 && TT == T && RR == R) ok = true;
#define OPO_HAS_WA(CC, TT, RR, RM)                                                                  \
    if (!tpass && (sizeof(CC) == 16) == fp64 && TT == T && RR == R) ok = true;
    OPO_WS_T_VARIANTS(OPO_HAS_WT)
    OPO_WS_A_VARIANTS(OPO_HAS_WA)
#undef OPO_HAS_WT
#undef OPO_HAS_WA
    return ok;
}

namespace {

template <typename C> const void *ws_fn(bool tpass, PassVariant v, bool bfast)
{
    const void *fn = nullptr;
#define OPO_FN_WT(CC, T, R, RM)                                                                     \
    if constexpr (std::is_same<C, CC>::value)                                                      \
        if (!fn && tpass && v.threads == T && v.r1 == R) fn = reinterpret_cast<const void *>(tpass_ws_kernel<CC, R, T, RM>);
#define OPO_FN_WA(CC, T, R, RM)                                                                     \
    if constexpr (std::is_same<C, CC>::value)                                                      \
        if (!fn && !tpass && v.threads == T && v.r1 == R)                                          \
            fn = bfast ? reinterpret_cast<const void *>(axis_ws_kernel<CC, R, true, T, RM>)        \
                       : reinterpret_cast<const void *>(axis_ws_kernel<CC, R, false, T, RM>);
    OPO_WS_T_VARIANTS(OPO_FN_WT)
    OPO_WS_A_VARIANTS(OPO_FN_WA)
#undef OPO_FN_WT
#undef OPO_FN_WA
    return fn;
}

}  // namespace

template <typename C> int ws_occupancy(bool tpass, PassVariant v, bool bfast, size_t smem)
{
    const void *fn = ws_fn<C>(tpass, v, bfast);
    int nb = 0;
    if (!fn || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, v.threads + 32, smem) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return nb;
}

template <typename C>
cudaError_t launch_tpass_ws(const TPassArgs<C> &a, const WsArgs &w, const CUtensorMap *maps, PassVariant v, int grid,
                            size_t smem, cudaStream_t st)
{
    const void *fn = ws_fn<C>(true, v, false);
    if (!fn) return cudaErrorInvalidValue;
    void *args[5] = {const_cast<TPassArgs<C> *>(&a), const_cast<WsArgs *>(&w), const_cast<CUtensorMap *>(&maps[0]),
                     const_cast<CUtensorMap *>(&maps[1]), const_cast<CUtensorMap *>(&maps[2])};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)(v.threads + 32)), args, smem, st);
}

template <typename C>
cudaError_t launch_axis_ws(const AxisArgs<C> &a, const WsArgs &w, const CUtensorMap *maps, PassVariant v, bool bfast,
                           int grid, size_t smem, cudaStream_t st)
{
    const void *fn = ws_fn<C>(false, v, bfast);
    if (!fn) return cudaErrorInvalidValue;
    void *args[5] = {const_cast<AxisArgs<C> *>(&a), const_cast<WsArgs *>(&w), const_cast<CUtensorMap *>(&maps[0]),
                     const_cast<CUtensorMap *>(&maps[1]), const_cast<CUtensorMap *>(&maps[2])};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3((unsigned)(v.threads + 32)), args, smem, st);
}

template int ws_occupancy<float2>(bool, PassVariant, bool, size_t);
template int ws_occupancy<double2>(bool, PassVariant, bool, size_t);
template cudaError_t launch_tpass_ws<float2>(const TPassArgs<float2> &, const WsArgs &, const CUtensorMap *, PassVariant,
                                             int, size_t, cudaStream_t);
template cudaError_t launch_tpass_ws<double2>(const TPassArgs<double2> &, const WsArgs &, const CUtensorMap *,
                                              PassVariant, int, size_t, cudaStream_t);
template cudaError_t launch_axis_ws<float2>(const AxisArgs<float2> &, const WsArgs &, const CUtensorMap *, PassVariant,
                                            bool, int, size_t, cudaStream_t);
template cudaError_t launch_axis_ws<double2>(const AxisArgs<double2> &, const WsArgs &, const CUtensorMap *,
                                             PassVariant, bool, int, size_t, cudaStream_t);

}  // namespace opo
