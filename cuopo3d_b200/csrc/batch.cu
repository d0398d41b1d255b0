// Batched split-step: many OPO instances (uneven grids and parameters) advance together,
// one persistent launch per pass covering the tiles of every instance.
//
// Each instance lives in a slot that owns a single-instance solver (its resident
// fields, FFT plans and phase tables, built with the batch's kernel variants).  The
// pass arguments of every active slot are kept in device descriptor arrays, with a
// tile-prefix array and a header {instances, tiles} per pass kind; a CTA of a batched
// kernel walks global tile numbers, finds the owning instance by binary search on the
// prefix array and stages that instance's descriptor in shared memory.  Because the
// instance list lives in device memory, the round trip is captured once as a CUDA graph
// and stays valid while slots are admitted and retired between round trips.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "pass_body.cuh"
#include "tpass_line.cuh"
#include "solver_internal.h"

namespace opo {

// One launch's share of a descriptor array: instances [first, first + ninst) with their
// tile prefix at prefix[pfirst ...] (starting at 0), total_tiles tiles.
struct BatchHeader {
    unsigned ninst;
    unsigned total_tiles;
    unsigned first;
    unsigned pfirst;
};

template <typename Args> __host__ __device__ constexpr unsigned desc_bytes() { return (unsigned)((sizeof(Args) + 127) / 128 * 128); }

template <typename Args> __device__ __forceinline__ void stage_desc(const Args *src, Args *dst)
{
    const unsigned *s = reinterpret_cast<const unsigned *>(src);
    unsigned *d = reinterpret_cast<unsigned *>(dst);
    for (unsigned k = threadIdx.x; k < sizeof(Args) / 4; k += blockDim.x) d[k] = s[k];
}

// Largest i < ninst with prefix[i] <= gt.
__device__ __forceinline__ int find_inst(const unsigned *prefix, unsigned ninst, unsigned gt)
{
    int lo = 0, hi = (int)ninst - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= gt) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename C, int R1, int THREADS, int RMAX>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 4 : 1)
    tpass_batch_kernel(const TPassArgs<C> *descs, const unsigned *prefix, const BatchHeader *hdr, int tp)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TPassArgs<C> *d = reinterpret_cast<TPassArgs<C> *>(smem_raw);
    C *sm = reinterpret_cast<C *>(smem_raw + desc_bytes<TPassArgs<C>>());
    const unsigned ninst = hdr->ninst, total = hdr->total_tiles;
    descs += hdr->first;
    prefix += hdr->pfirst;
    int cur = -1;
    for (unsigned gt = blockIdx.x; gt < total; gt += gridDim.x) {
        const int i = find_inst(prefix, ninst, gt);
        if (i != cur) {
            __syncthreads();
            stage_desc(descs + i, d);
            __syncthreads();
            if (threadIdx.x < 6 && d->ph_steps) d->ph[threadIdx.x / 3][threadIdx.x % 3] = d->ph_steps[tp * 6 + threadIdx.x];
            __syncthreads();
            cur = i;
        }
        // stage the tile with cp.async first, as the single-instance t-pass does
        const unsigned tile = gt - __ldg(prefix + i);
        const C *src[3] = {d->psrc, d->f[1], d->f[2]};
        stage_tile<C, THREADS, false>(d->g, (unsigned)d->plan.n, tile, src, tpass_load_mask(*d), sm);
        tpass_tile<C, R1, THREADS, RMAX, true>(*d, tile, sm);
    }
}

// Batched line-specialised t-pass for the instances whose time axis has the line body
// (NT, RA): one tile at a time, one tile buffer.  Each line body has a kernel of its own
// (one kernel holding every body and the generic one needed 168 registers and spilled);
// the instances without a line body run tpass_batch_kernel with the fallback radix.
template <typename C, int NT, int RA, int THREADS>
__global__ void __launch_bounds__(THREADS, 4)
    tpass_line_batch_kernel(const TPassArgs<C> *descs, const unsigned *prefix, const BatchHeader *hdr, int tp)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TPassArgs<C> *d = reinterpret_cast<TPassArgs<C> *>(smem_raw);
    unsigned char *buf = smem_raw + desc_bytes<TPassArgs<C>>();
    const unsigned ninst = hdr->ninst, total = hdr->total_tiles;
    descs += hdr->first;
    prefix += hdr->pfirst;
    int cur = -1;
    for (unsigned gt = blockIdx.x; gt < total; gt += gridDim.x) {
        const int i = find_inst(prefix, ninst, gt);
        if (i != cur) {
            __syncthreads();
            stage_desc(descs + i, d);
            __syncthreads();
            if (threadIdx.x < 6 && d->ph_steps) d->ph[threadIdx.x / 3][threadIdx.x % 3] = d->ph_steps[tp * 6 + threadIdx.x];
            __syncthreads();
            cur = i;
        }
        tpass_line_tile<C, NT, RA, THREADS>(*d, gt - __ldg(prefix + i), buf);
    }
}

template <typename C, int R1, bool BFAST, int THREADS, int RMAX>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 4 : 1)
    axis_batch_kernel(const AxisArgs<C> *descs, const unsigned *prefix, const BatchHeader *hdr)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    AxisArgs<C> *d = reinterpret_cast<AxisArgs<C> *>(smem_raw);
    C *sm = reinterpret_cast<C *>(smem_raw + desc_bytes<AxisArgs<C>>());
    const unsigned ninst = hdr->ninst, total = hdr->total_tiles;
    descs += hdr->first;
    prefix += hdr->pfirst;
    int cur = -1;
    for (unsigned gt = blockIdx.x; gt < total; gt += gridDim.x) {
        const int i = find_inst(prefix, ninst, gt);
        if (i != cur) {
            __syncthreads();
            stage_desc(descs + i, d);
            __syncthreads();
            cur = i;
        }
        axis_tile<C, R1, BFAST, THREADS, RMAX>(*d, gt - __ldg(prefix + i), sm);
    }
}

// FP64 sums of |A|^2 of every active slot: block (bx, slot) reduces a strided share of
// the slot's three fields into partials[slot][bx]; one thread per slot and field then
// adds the partials in a fixed order.
struct SlotFields {
    const void *f[3];
    unsigned long long n;
};

constexpr int kTallyThreads = 256;
constexpr int kTallyBlocks = 64;  // per slot

template <typename C>
__global__ void __launch_bounds__(kTallyThreads) batch_tally_kernel(const SlotFields *sf, double *partials)
{
    __shared__ double red[3][kTallyThreads / 32];
    const SlotFields s = sf[blockIdx.y];
    double acc[3] = {0, 0, 0};
    for (unsigned long long v = (unsigned long long)blockIdx.x * kTallyThreads + threadIdx.x; v < s.n;
         v += (unsigned long long)kTallyBlocks * kTallyThreads) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const C a = static_cast<const C *>(s.f[k])[v];
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
        for (int w = 0; w < kTallyThreads / 32; w++) x += red[threadIdx.x][w];
        partials[((size_t)blockIdx.y * kTallyBlocks + blockIdx.x) * 3 + threadIdx.x] = x;
    }
}

__global__ void batch_tally_final_kernel(const double *partials, int nslots, double *out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nslots * 3) return;
    const int slot = t / 3, k = t % 3;
    double x = 0;
    for (int b = 0; b < kTallyBlocks; b++) x += partials[((size_t)slot * kTallyBlocks + b) * 3 + k];
    out[t] = x;
}

// ---------------------------------------------------------------------------------
// Compiled batched variants (the same set as the single-instance kernels).

#define OPO_BT_VARIANTS(X)                                                                         \
    X(float2, 128, 4, 16) X(float2, 128, 8, 16) X(float2, 128, 16, 16) X(float2, 256, 4, 16)        \
    X(float2, 256, 8, 16) X(float2, 256, 16, 16) X(double2, 128, 4, 8) X(double2, 128, 8, 8)        \
    X(double2, 256, 4, 16) X(double2, 256, 8, 16)

#define OPO_BA_VARIANTS(X)                                                                         \
    X(float2, 128, 4, 16) X(float2, 128, 8, 16) X(float2, 128, 16, 16) X(float2, 256, 4, 16)        \
    X(float2, 256, 8, 16) X(float2, 256, 16, 16) X(double2, 128, 4, 8) X(double2, 128, 8, 8)        \
    X(double2, 256, 4, 16) X(double2, 256, 8, 16) X(double2, 256, 16, 16)

// t-pass groups: under the line-specialised setting, the instances with the 256-, 128-
// and 64-sample line bodies (groups 0-2) and the rest (group 3, the generic body with the
// fallback radix); under any other setting every instance is in group 3.
constexpr int kTGroups = 4;
inline int t_group(PassVariant v, int line_nt)
{
    if (!is_line(v)) return 3;
    return line_nt == 256 ? 0 : line_nt == 128 ? 1 : line_nt == 64 ? 2 : 3;
}
constexpr int kLineGroupNT[3] = {256, 128, 64};

template <typename C> bool batch_t_generic_func(PassVariant v, const void **fn);

// Resolves the batched kernel of each t-pass group (nullptr: the group is never
// populated under this setting); returns false if a variant is not compiled.
template <typename C> bool batch_t_funcs(PassVariant v, const void *fn[kTGroups])
{
    for (int g = 0; g < kTGroups; g++) fn[g] = nullptr;
    if (!is_line(v)) return batch_t_generic_func<C>(v, &fn[3]);
    if (v.threads != 128 || !line_variant_compiled(v.threads, radix_of(v))) return false;
    fn[0] = reinterpret_cast<const void *>(tpass_line_batch_kernel<C, 256, 16, 128>);
    fn[1] = reinterpret_cast<const void *>(tpass_line_batch_kernel<C, 128, 16, 128>);
    fn[2] = reinterpret_cast<const void *>(tpass_line_batch_kernel<C, 64, 8, 128>);
    return batch_t_generic_func<C>(PassVariant{128, line_fallback_radix(sizeof(C) == 16, v)}, &fn[3]);
}

template <typename C> bool batch_t_generic_func(PassVariant v, const void **fn)
{
    bool ok = false;
#define OPO_F_T(CC, T, R, RM)                                                                       \
    if constexpr (std::is_same<C, CC>::value) {                                                     \
        if (!ok && v.threads == T && v.r1 == R) {                                                   \
            *fn = reinterpret_cast<const void *>(tpass_batch_kernel<CC, R, T, RM>);                 \
            ok = true;                                                                              \
        }                                                                                           \
    }
    OPO_BT_VARIANTS(OPO_F_T)
#undef OPO_F_T
    return ok;
}

template <typename C> bool batch_a_func(PassVariant v, bool bfast, const void **fn)
{
    bool ok = false;
#define OPO_F_A(CC, T, R, RM)                                                                       \
    if constexpr (std::is_same<C, CC>::value) {                                                     \
        if (!ok && v.threads == T && v.r1 == R) {                                                   \
            *fn = bfast ? reinterpret_cast<const void *>(axis_batch_kernel<CC, R, true, T, RM>)      \
                        : reinterpret_cast<const void *>(axis_batch_kernel<CC, R, false, T, RM>);   \
            ok = true;                                                                              \
        }                                                                                           \
    }
    OPO_BA_VARIANTS(OPO_F_A)
#undef OPO_F_A
    return ok;
}

}  // namespace opo

// =================================================================================
// Host layer.

namespace {

using cd = std::complex<double>;

struct Slot {
    bool used = false;
    OpoSolver *s = nullptr;
    int rt = 0;
    int total_rt = 1;
    size_t bytes = 0;
    void *ph_steps = nullptr;  // device [n_steps + 1][2][3] phases (corrected physics with dk)
    long long voxels = 0;
};

}  // namespace

struct OpoBatch {
    int precision = OPO_FP32;
    int capacity = 0;
    int n_steps = 0;
    int dev = 0;
    int sms = 148;
    size_t budget = 0, used = 0;
    opo::PassVariant v[3];
    size_t te[3];
    cudaStream_t stream = nullptr;
    std::vector<Slot> slots;
    std::vector<int> order;  // active slots in descriptor order
    // device state
    void *d_t[3] = {};       // t descriptors: first, middle, final
    void *d_ax[2][2] = {};   // [x, y][crystal, free]
    unsigned *d_prefix[3] = {};  // t: one prefix per t-pass group, back to back
    opo::BatchHeader *d_hdr = nullptr;  // [t-pass groups..., x, y]
    opo::SlotFields *d_slotf = nullptr;
    double *d_partials = nullptr, *d_sums = nullptr;
    std::vector<unsigned char> h_desc;  // host staging
    bool dirty = true;
    std::vector<char> last_flag;  // per order position: on its last round trip when uploaded
    cudaGraphExec_t graph = nullptr;
    size_t graph_smem[3] = {0, 0, 0};  // t: the generic group's
    int grid[3] = {0, 0, 0};
    int t_grid[opo::kTGroups] = {};
    size_t t_smem[opo::kTGroups] = {};
    long long launches = 0;
    int launches_rt = 0;
    std::string err;
};

namespace {

thread_local std::string g_batch_err;

int bfail(OpoBatch *b, int code, const std::string &msg)
{
    if (b) b->err = msg;
    else g_batch_err = msg;
    return code;
}

#define OPO_BCU(b, call, what)                                                                  \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? OPO_ERR_NOMEM : OPO_ERR_CUDA,   \
                         std::string(what) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

bool slot_ok(const OpoBatch *b, int slot) { return b && slot >= 0 && slot < b->capacity && b->slots[slot].used; }

template <typename C> int upload_descriptors(OpoBatch *b)
{
    using TA = opo::TPassArgs<C>;
    using AA = opo::AxisArgs<C>;
    const int n = (int)b->order.size();
    std::vector<TA> t[3];
    std::vector<AA> ax[2][2];
    std::vector<unsigned> prefix[3];
    std::vector<opo::SlotFields> sf;
    std::vector<int> tgroup;
    for (int k = 1; k < 3; k++) prefix[k].push_back(0);
    b->last_flag.assign(n, 0);
    for (int pos = 0; pos < n; pos++) {
        Slot &sl = b->slots[b->order[pos]];
        OpoSolver *s = sl.s;
        const OpoParams &p = opo::solver_params(s);
        const bool disp = (p.flags & OPO_DISPERSION) != 0, diff = (p.flags & OPO_DIFFRACTION) != 0;
        const bool last = sl.rt == sl.total_rt - 1;
        b->last_flag[pos] = last;
        double zh[2];
        int nrk;
        opo::solver_tpass_z(p, 0, zh, &nrk);
        t[0].push_back(opo::make_tpass_args<C>(s, true, nrk, zh, 0, disp ? 7u : 0u));
        opo::solver_tpass_z(p, p.n_steps > 1 ? 1 : 0, zh, &nrk);
        t[1].push_back(opo::make_tpass_args<C>(s, false, 2, zh, 0, disp ? 7u : 0u));
        opo::solver_tpass_z(p, p.n_steps, zh, &nrk);
        t[2].push_back(opo::make_tpass_args<C>(s, false, 1, zh, 1, opo::solver_gdd_or_mirror(s) ? 6u : 0u));
        for (int k = 0; k < 3; k++) t[k].back().ph_steps = static_cast<const C *>(sl.ph_steps);
        for (int a = 0; a < 2; a++) {
            ax[a][0].push_back(opo::make_axis_args<C>(s, 1 + a, 0, diff ? 7u : 0u));
            ax[a][1].push_back(opo::make_axis_args<C>(s, 1 + a, 1, (diff && !last) ? 6u : 0u));
        }
        tgroup.push_back(opo::t_group(b->v[0], opo::solver_line_nt(s)));
        for (int k = 1; k < 3; k++) {
            int nt;
            size_t sm;
            opo::solver_pass_info(s, k, &nt, &sm);
            prefix[k].push_back(prefix[k].back() + (unsigned)nt);
        }
        opo::SlotFields f;
        for (int k = 0; k < 3; k++) f.f[k] = opo::solver_field(s, k + 1);
        f.n = (unsigned long long)sl.voxels;
        sf.push_back(f);
    }
    // t descriptors group-major, each group with its own tile prefix (from 0)
    opo::BatchHeader hdr[opo::kTGroups + 2];
    {
        std::vector<TA> ts[3];
        for (int g = 0; g < opo::kTGroups; g++) {
            hdr[g].first = (unsigned)ts[0].size();
            hdr[g].pfirst = (unsigned)prefix[0].size();
            prefix[0].push_back(0);
            for (int pos = 0; pos < n; pos++) {
                if (tgroup[pos] != g) continue;
                for (int k = 0; k < 3; k++) ts[k].push_back(t[k][pos]);
                int nt;
                size_t sm;
                opo::solver_pass_info(b->slots[b->order[pos]].s, 0, &nt, &sm);
                prefix[0].push_back(prefix[0].back() + (unsigned)nt);
            }
            hdr[g].ninst = (unsigned)ts[0].size() - hdr[g].first;
            hdr[g].total_tiles = prefix[0].back();
        }
        for (int k = 0; k < 3; k++) t[k].swap(ts[k]);
    }
    const size_t cap = (size_t)b->capacity;
    for (int k = 0; k < 3; k++)
        if (n) OPO_BCU(b, cudaMemcpyAsync(b->d_t[k], t[k].data(), sizeof(TA) * n, cudaMemcpyHostToDevice, b->stream), "descriptors");
    for (int a = 0; a < 2; a++)
        for (int w = 0; w < 2; w++)
            if (n) OPO_BCU(b, cudaMemcpyAsync(b->d_ax[a][w], ax[a][w].data(), sizeof(AA) * n, cudaMemcpyHostToDevice, b->stream), "descriptors");
    for (int k = 0; k < 3; k++)
        OPO_BCU(b, cudaMemcpyAsync(b->d_prefix[k], prefix[k].data(), sizeof(unsigned) * prefix[k].size(),
                                   cudaMemcpyHostToDevice, b->stream), "prefix");
    for (int a = 0; a < 2; a++) hdr[opo::kTGroups + a] = opo::BatchHeader{(unsigned)n, prefix[1 + a].back(), 0, 0};
    OPO_BCU(b, cudaMemcpyAsync(b->d_hdr, hdr, sizeof(hdr), cudaMemcpyHostToDevice, b->stream), "header");
    if (n) OPO_BCU(b, cudaMemcpyAsync(b->d_slotf, sf.data(), sizeof(opo::SlotFields) * n, cudaMemcpyHostToDevice, b->stream), "slot fields");
    // pageable sources: make the copies complete before the host vectors go away
    OPO_BCU(b, cudaStreamSynchronize(b->stream), "descriptor sync");
    (void)cap;
    b->dirty = false;
    return OPO_OK;
}

// Persistent grid of a batched kernel: SMs x resident CTAs at this shared-memory size.
int persistent_grid(OpoBatch *b, const void *fn, int threads, size_t smem)
{
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess || per < 1) per = 1;
    return b->sms * per;
}

template <typename C> int enqueue_batch_round_trip(OpoBatch *b)
{
    using TA = opo::TPassArgs<C>;
    using AA = opo::AxisArgs<C>;
    const void *ft[opo::kTGroups], *fx = nullptr, *fy = nullptr;
    if (!opo::batch_t_funcs<C>(b->v[0], ft) || !opo::batch_a_func<C>(b->v[1], true, &fx) ||
        !opo::batch_a_func<C>(b->v[2], false, &fy))
        return bfail(b, OPO_ERR_INVALID, "batch kernel variant not compiled");
    const size_t sx = opo::desc_bytes<AA>() + b->graph_smem[1];
    const size_t sy = opo::desc_bytes<AA>() + b->graph_smem[2];
    const opo::BatchHeader *hdr = b->d_hdr;
    // one launch per t-pass group the setting populates; a group without instances
    // (its header counts none) returns at once
    auto launch_t = [&](int which, int tp) -> cudaError_t {
        const TA *descs = static_cast<const TA *>(b->d_t[which]);
        const unsigned *pre = b->d_prefix[0];
        for (int g = 0; g < opo::kTGroups; g++) {
            if (!ft[g]) continue;
            const opo::BatchHeader *h = hdr + g;
            void *args[] = {(void *)&descs, (void *)&pre, (void *)&h, (void *)&tp};
            b->launches++;
            cudaError_t e = cudaLaunchKernel(ft[g], dim3(b->t_grid[g]), dim3(b->v[0].threads), args, b->t_smem[g],
                                             b->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    auto launch_a = [&](int axis, int which) -> cudaError_t {
        const AA *descs = static_cast<const AA *>(b->d_ax[axis][which]);
        const unsigned *pre = b->d_prefix[1 + axis];
        const opo::BatchHeader *h = hdr + opo::kTGroups + axis;
        void *args[] = {(void *)&descs, (void *)&pre, (void *)&h};
        b->launches++;
        return cudaLaunchKernel(axis == 0 ? fx : fy, dim3(b->grid[1 + axis]), dim3(b->v[1 + axis].threads), args,
                                axis == 0 ? sx : sy, b->stream);
    };
    for (int k = 0; k < b->n_steps; k++) {
        OPO_BCU(b, launch_t(k == 0 ? 0 : 1, k), "batch t-pass");
        OPO_BCU(b, launch_a(0, 0), "batch x-pass");
        OPO_BCU(b, launch_a(1, 0), "batch y-pass");
    }
    OPO_BCU(b, launch_t(2, b->n_steps), "batch t-pass");
    OPO_BCU(b, launch_a(0, 1), "batch x-pass");
    OPO_BCU(b, launch_a(1, 1), "batch y-pass");
    return OPO_OK;
}

template <typename C> int build_batch_graph(OpoBatch *b)
{
    using TA = opo::TPassArgs<C>;
    using AA = opo::AxisArgs<C>;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    // shared memory: the largest tile of any slot, per pass kind (t: of the slots in the
    // generic group; a line body's tile has a fixed size)
    for (int k = 0; k < 3; k++) b->graph_smem[k] = 0;
    for (int sidx : b->order) {
        for (int k = 0; k < 3; k++) {
            int nt;
            size_t sm;
            opo::solver_pass_info(b->slots[sidx].s, k, &nt, &sm);
            if (k == 0 && opo::t_group(b->v[0], opo::solver_line_nt(b->slots[sidx].s)) != 3) continue;
            b->graph_smem[k] = std::max(b->graph_smem[k], sm);
        }
    }
    const void *ft[opo::kTGroups], *fx = nullptr, *fy = nullptr;
    if (!opo::batch_t_funcs<C>(b->v[0], ft) || !opo::batch_a_func<C>(b->v[1], true, &fx) ||
        !opo::batch_a_func<C>(b->v[2], false, &fy))
        return bfail(b, OPO_ERR_INVALID, "batch kernel variant not compiled");
    const bool fp64 = sizeof(C) == 16;
    for (int g = 0; g < opo::kTGroups; g++) {
        if (!ft[g]) continue;
        b->t_smem[g] = opo::desc_bytes<TA>() +
                       (g < 3 ? opo::tpass_line_smem(fp64, opo::kLineGroupNT[g], opo::line_radix(opo::kLineGroupNT[g]))
                              : b->graph_smem[0]);
        if (b->t_smem[g] > 227 * 1024) return bfail(b, OPO_ERR_INVALID, "batched tile does not fit in shared memory");
        OPO_BCU(b, cudaFuncSetAttribute(ft[g], cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "attribute");
        b->t_grid[g] = persistent_grid(b, ft[g], b->v[0].threads, b->t_smem[g]);
    }
    const size_t sm[3] = {0, opo::desc_bytes<AA>() + b->graph_smem[1], opo::desc_bytes<AA>() + b->graph_smem[2]};
    const void *fns[3] = {nullptr, fx, fy};
    for (int k = 1; k < 3; k++) {
        if (sm[k] > 227 * 1024) return bfail(b, OPO_ERR_INVALID, "batched tile does not fit in shared memory");
        OPO_BCU(b, cudaFuncSetAttribute(fns[k], cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024), "attribute");
        b->grid[k] = persistent_grid(b, fns[k], b->v[k].threads, sm[k]);
    }
    cudaGraph_t g = nullptr;
    OPO_BCU(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    const long long before = b->launches;
    int rc = enqueue_batch_round_trip<C>(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return bfail(b, OPO_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
    b->launches_rt = (int)(b->launches - before);
    b->launches = before;
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bfail(b, OPO_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return OPO_OK;
}

template <typename C> int batch_run(OpoBatch *b, int n)
{
    for (int r = 0; r < n; r++) {
        if (b->order.empty()) return OPO_OK;
        bool need = b->dirty;
        for (size_t pos = 0; pos < b->order.size() && !need; pos++) {
            const Slot &sl = b->slots[b->order[pos]];
            need = (sl.rt == sl.total_rt - 1) != (b->last_flag[pos] != 0);
        }
        if (need) {
            int rc = upload_descriptors<C>(b);
            if (rc) return rc;
        }
        bool rebuild = !b->graph;
        for (int sidx : b->order)
            for (int k = 0; k < 3; k++) {
                int nt;
                size_t sm;
                opo::solver_pass_info(b->slots[sidx].s, k, &nt, &sm);
                if (k == 0 && opo::t_group(b->v[0], opo::solver_line_nt(b->slots[sidx].s)) != 3) continue;
                if (sm > b->graph_smem[k]) rebuild = true;
            }
        if (rebuild) {
            int rc = build_batch_graph<C>(b);
            if (rc) return rc;
        }
        OPO_BCU(b, cudaGraphLaunch(b->graph, b->stream), "batch graph launch");
        b->launches += b->launches_rt;
        for (int sidx : b->order) b->slots[sidx].rt++;
    }
    return OPO_OK;
}

template <typename C> int batch_sums(OpoBatch *b, double *out)
{
    const int n = (int)b->order.size();
    for (int k = 0; k < 3 * b->capacity; k++) out[k] = 0;
    if (!n) return OPO_OK;
    if (b->dirty) {
        int rc = upload_descriptors<C>(b);
        if (rc) return rc;
    }
    opo::batch_tally_kernel<C><<<dim3(opo::kTallyBlocks, n), opo::kTallyThreads, 0, b->stream>>>(b->d_slotf, b->d_partials);
    opo::batch_tally_final_kernel<<<(3 * n + 127) / 128, 128, 0, b->stream>>>(b->d_partials, n, b->d_sums);
    OPO_BCU(b, cudaGetLastError(), "batch tallies");
    b->launches += 2;
    std::vector<double> h(3 * n);
    OPO_BCU(b, cudaMemcpyAsync(h.data(), b->d_sums, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, b->stream), "tallies copy");
    OPO_BCU(b, cudaStreamSynchronize(b->stream), "tallies sync");
    for (int pos = 0; pos < n; pos++)
        for (int k = 0; k < 3; k++) out[3 * b->order[pos] + k] = h[3 * pos + k];
    return OPO_OK;
}

}  // namespace

// =================================================================================
// C-ABI

extern "C" {

int opo_batch_create(int precision, int capacity, size_t hbm_budget, const int tuning[9], OpoBatch **out)
{
    if (!out) return OPO_ERR_INVALID;
    *out = nullptr;
    if ((precision != OPO_FP32 && precision != OPO_FP64) || capacity < 1 || capacity > 65536)
        return bfail(nullptr, OPO_ERR_INVALID, "opo_batch_create: bad precision or capacity");
    OpoBatch *b = new (std::nothrow) OpoBatch();
    if (!b) return OPO_ERR_NOMEM;
    b->precision = precision;
    b->capacity = capacity;
    b->budget = hbm_budget;
    b->slots.resize(capacity);
    const bool fp64 = precision == OPO_FP64;
    for (int k = 0; k < 3; k++) {
        if (tuning) {
            // the batched kernels have no warp-specialised form: a warp-specialised CTA
            // size (160 / 288) runs as its consumer size (128 / 256)
            b->v[k] = opo::PassVariant{opo::consumer_threads(opo::PassVariant{tuning[3 * k], 0}), tuning[3 * k + 2]};
            b->te[k] = (size_t)tuning[3 * k + 1];
        } else {
            b->v[k] = opo::PassVariant{128, k == 0 ? 4 : 8};
            b->te[k] = fp64 ? 1024 : 2048;
        }
        if (!opo::variant_compiled(fp64, k == 0, b->v[k])) {
            delete b;
            return bfail(nullptr, OPO_ERR_INVALID, "opo_batch_create: kernel variant not compiled");
        }
    }
    int rc = OPO_OK;
    cudaError_t e = cudaSuccess;
    do {
        if ((e = cudaGetDevice(&b->dev)) != cudaSuccess) { rc = OPO_ERR_CUDA; break; }
        cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->dev);
        if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = OPO_ERR_CUDA; break; }
        const size_t tsz = fp64 ? sizeof(opo::TPassArgs<double2>) : sizeof(opo::TPassArgs<float2>);
        const size_t asz = fp64 ? sizeof(opo::AxisArgs<double2>) : sizeof(opo::AxisArgs<float2>);
        for (int k = 0; k < 3 && !rc; k++)
            if (cudaMalloc(&b->d_t[k], tsz * capacity) != cudaSuccess) rc = OPO_ERR_NOMEM;
        for (int a = 0; a < 2 && !rc; a++)
            for (int w = 0; w < 2 && !rc; w++)
                if (cudaMalloc(&b->d_ax[a][w], asz * capacity) != cudaSuccess) rc = OPO_ERR_NOMEM;
        for (int k = 0; k < 3 && !rc; k++)
            if (cudaMalloc((void **)&b->d_prefix[k], sizeof(unsigned) * (capacity + opo::kTGroups)) != cudaSuccess)
                rc = OPO_ERR_NOMEM;
        if (rc) break;
        if (cudaMalloc((void **)&b->d_hdr, sizeof(opo::BatchHeader) * (opo::kTGroups + 2)) != cudaSuccess ||
            cudaMalloc((void **)&b->d_slotf, sizeof(opo::SlotFields) * capacity) != cudaSuccess ||
            cudaMalloc((void **)&b->d_partials, sizeof(double) * 3 * opo::kTallyBlocks * capacity) != cudaSuccess ||
            cudaMalloc((void **)&b->d_sums, sizeof(double) * 3 * capacity) != cudaSuccess) {
            rc = OPO_ERR_NOMEM;
            break;
        }
    } while (0);
    if (rc) {
        opo_batch_destroy(b);
        return bfail(nullptr, rc, std::string("opo_batch_create: device set-up failed: ") + cudaGetErrorString(e));
    }
    *out = b;
    return OPO_OK;
}

void opo_batch_destroy(OpoBatch *b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto &sl : b->slots) {
        if (sl.s) opo_destroy(sl.s);
        if (sl.ph_steps) cudaFree(sl.ph_steps);
    }
    for (auto *p : b->d_t) cudaFree(p);
    for (auto &row : b->d_ax)
        for (auto *p : row) cudaFree(p);
    for (auto *p : b->d_prefix) cudaFree(p);
    cudaFree(b->d_hdr);
    cudaFree(b->d_slotf);
    cudaFree(b->d_partials);
    cudaFree(b->d_sums);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int opo_batch_add(OpoBatch *b, const OpoParams *p, const double *w, int *slot_out)
{
    if (!b || !p || !w || !slot_out) return OPO_ERR_INVALID;
    *slot_out = -1;
    if (p->precision != b->precision) return bfail(b, OPO_ERR_INVALID, "instance precision differs from the batch");
    // every resident instance takes the same number of z-steps (one round-trip graph);
    // an instance with another count waits until the batch has drained
    if (!b->order.empty() && p->n_steps != b->n_steps)
        return bfail(b, OPO_ERR_CAPACITY, "the resident instances take another number of z-steps");
    int free_slot = -1;
    for (int k = 0; k < b->capacity; k++)
        if (!b->slots[k].used) { free_slot = k; break; }
    if (free_slot < 0) return bfail(b, OPO_ERR_CAPACITY, "no free slot");
    const size_t esz = b->precision == OPO_FP64 ? 16 : 8;
    const size_t V = (size_t)p->nx * p->ny * p->nt;
    const size_t need = opo::batch_instance_bytes(b->precision, V);  // fields + tables and plans
    if (b->used + need > b->budget) return bfail(b, OPO_ERR_CAPACITY, "HBM budget exhausted");
    OpoSolver *s = nullptr;
    int rc = opo::solver_create_configured(p, w, b->v, b->te, b->stream, &s);
    if (rc) return bfail(b, rc, "instance creation failed (grid not supported by the batch's kernel variants?)");
    for (int k = 0; k < 3; k++) {
        const opo::PassVariant got = opo::solver_pass_variant(s, k);
        if (got.r1 != b->v[k].r1 || got.threads != b->v[k].threads || (k == 0 && !opo::solver_line_fallback_ok(s))) {
            opo_destroy(s);
            return bfail(b, OPO_ERR_INVALID, "grid needs a first-stage radix other than the batch's");
        }
    }
    Slot &sl = b->slots[free_slot];
    sl = Slot{};
    sl.used = true;
    sl.s = s;
    sl.rt = 0;
    sl.total_rt = p->total_rt > 0 ? p->total_rt : 1;
    sl.bytes = need;
    sl.voxels = (long long)V;
    if ((p->flags & OPO_PHYSICS) && p->dk != 0) {
        // phases exp(i dk z) of every t-pass of a round trip, [tp][half][stage]
        std::vector<cd> ph((size_t)(p->n_steps + 1) * 6);
        const double h = 0.5 * p->dz;
        for (int tp = 0; tp <= p->n_steps; tp++) {
            double zh[2];
            int nrk;
            opo::solver_tpass_z(*p, tp, zh, &nrk);
            for (int k = 0; k < 2; k++) {
                const double zs[3] = {zh[k], zh[k] + 0.5 * h, zh[k] + h};
                for (int j = 0; j < 3; j++) ph[(size_t)tp * 6 + k * 3 + j] = std::polar(1.0, p->dk * zs[j]);
            }
        }
        const size_t bytes = ph.size() * esz;
        if (cudaMalloc(&sl.ph_steps, bytes) != cudaSuccess) {
            opo_destroy(s);
            sl = Slot{};
            return bfail(b, OPO_ERR_NOMEM, "phase table allocation");
        }
        std::vector<unsigned char> buf(bytes);
        for (size_t k = 0; k < ph.size(); k++) {
            if (esz == 16) {
                const double2 v = make_double2(ph[k].real(), ph[k].imag());
                std::memcpy(&buf[k * esz], &v, esz);
            } else {
                const float2 v = make_float2((float)ph[k].real(), (float)ph[k].imag());
                std::memcpy(&buf[k * esz], &v, esz);
            }
        }
        cudaMemcpy(sl.ph_steps, buf.data(), bytes, cudaMemcpyHostToDevice);
    }
    if (b->order.empty()) b->n_steps = p->n_steps;
    b->order.push_back(free_slot);
    b->used += need;
    b->dirty = true;
    *slot_out = free_slot;
    return OPO_OK;
}

int opo_batch_remove(OpoBatch *b, int slot)
{
    if (!slot_ok(b, slot)) return b ? bfail(b, OPO_ERR_INVALID, "bad slot") : OPO_ERR_INVALID;
    Slot &sl = b->slots[slot];
    cudaStreamSynchronize(b->stream);
    opo_destroy(sl.s);
    if (sl.ph_steps) cudaFree(sl.ph_steps);
    b->used -= sl.bytes;
    sl = Slot{};
    b->order.erase(std::remove(b->order.begin(), b->order.end(), slot), b->order.end());
    b->dirty = true;
    return OPO_OK;
}

int opo_batch_set_field(OpoBatch *b, int slot, int which, const void *src, int where, int prec)
{
    if (!slot_ok(b, slot)) return b ? bfail(b, OPO_ERR_INVALID, "bad slot") : OPO_ERR_INVALID;
    int rc = opo_set_field(b->slots[slot].s, which, src, where, prec);
    if (rc) return bfail(b, rc, opo_last_error(b->slots[slot].s));
    opo::solver_release_staging(b->slots[slot].s);  // keep the slot within its charge
    return OPO_OK;
}

int opo_batch_get_field(OpoBatch *b, int slot, int which, void *dst, int where, int prec)
{
    if (!slot_ok(b, slot)) return b ? bfail(b, OPO_ERR_INVALID, "bad slot") : OPO_ERR_INVALID;
    int rc = opo_get_field(b->slots[slot].s, which, dst, where, prec);
    if (rc) return bfail(b, rc, opo_last_error(b->slots[slot].s));
    opo::solver_release_staging(b->slots[slot].s);
    return OPO_OK;
}

int opo_batch_init_fields(OpoBatch *b, int slot, const OpoConfig *cfg, uint64_t seed, double sigma, int idler_copy)
{
    if (!slot_ok(b, slot) || !cfg) return b ? bfail(b, OPO_ERR_INVALID, "bad slot or configuration") : OPO_ERR_INVALID;
    int rc = opo::init_fields_device(b->slots[slot].s, cfg, seed, sigma, idler_copy, b->stream);
    if (rc) return bfail(b, rc, opo_last_error(b->slots[slot].s));
    b->launches++;
    return OPO_OK;
}

int opo_batch_run_round_trips(OpoBatch *b, int n)
{
    if (!b || n < 0) return OPO_ERR_INVALID;
    return b->precision == OPO_FP64 ? batch_run<double2>(b, n) : batch_run<float2>(b, n);
}

int opo_batch_sums(OpoBatch *b, double *sums)
{
    if (!b || !sums) return OPO_ERR_INVALID;
    return b->precision == OPO_FP64 ? batch_sums<double2>(b, sums) : batch_sums<float2>(b, sums);
}

int opo_batch_info(const OpoBatch *b, int slot, long long out[4])
{
    if (!slot_ok(b, slot) || !out) return OPO_ERR_INVALID;
    const Slot &sl = b->slots[slot];
    out[0] = sl.rt;
    out[1] = sl.total_rt;
    out[2] = sl.voxels;
    out[3] = (long long)sl.bytes;
    return OPO_OK;
}

int opo_batch_stats(const OpoBatch *b, long long out[4])
{
    if (!b || !out) return OPO_ERR_INVALID;
    out[0] = (long long)b->order.size();
    out[1] = (long long)b->used;
    out[2] = (long long)b->budget;
    out[3] = b->launches;
    return OPO_OK;
}

int opo_batch_get_stream(const OpoBatch *b, void **stream)
{
    if (!b || !stream) return OPO_ERR_INVALID;
    *stream = (void *)b->stream;
    return OPO_OK;
}

int opo_batch_synchronize(OpoBatch *b)
{
    if (!b) return OPO_ERR_INVALID;
    OPO_BCU(b, cudaStreamSynchronize(b->stream), "synchronize");
    return OPO_OK;
}

const char *opo_batch_last_error(const OpoBatch *b) { return b ? b->err.c_str() : g_batch_err.c_str(); }

}  // extern "C"
