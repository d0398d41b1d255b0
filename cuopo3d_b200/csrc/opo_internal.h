// Internal types shared by the host schedule (opo_host.cu) and the pass kernels
// (ssfm_kernels.cu).  Not part of the C-ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

namespace opo {

constexpr int kMaxStages = 8;

// Division by a run-time invariant d for n < 2^31 with one multiply-high and a shift
// (Granlund & Montgomery, "Division by invariant integers using multiplication", 1994):
// q = (m ? umulhi(n, m) : n) >> s, with m = ceil(2^(31+l) / d), s = l - 1, l = ceil(log2 d)
// for d not a power of two, and m = 0, s = log2 d otherwise.
struct FastDiv {
    unsigned d, m, s;
};

#ifdef __CUDACC__
__device__ __forceinline__ unsigned fdiv(const FastDiv &f, unsigned n)
{
    return (f.m ? __umulhi(n, f.m) : n) >> f.s;
}
#endif

// In-place line FFT of length n done in `ns` stages.  Forward stages are decimation in
// frequency: stage s splits sub-sequences of length len[s] with radix radix[s]
// (len[0] = n, len[s+1] = len[s] / radix[s], len[ns-1] = radix[ns-1]); the output is
// in mixed-radix digit-reversed order, which the phase tables are permuted to match,
// and the inverse stages (decimation in time, reverse order) restore natural order.
// Stage s twiddles W_len^{j k} = exp(-2 pi i j k / len) sit at tw[twoff[s] + (k-1) q + j],
// q = len / radix, k in [1, radix), j in [0, q).
struct AxisPlan {
    int n;
    int ns;
    int radix[kMaxStages];
    int len[kMaxStages];
    int twoff[kMaxStages];
    FastDiv q[kMaxStages];  // len[s] / radix[s]
};

// Placement of one tile of lines.  Line l, element j of tile `tile` is the global
// element  base(tile) + j * gs_j + l * gs_l  with
//   base(tile) = (tile % tdiv) * tmulA + (tile / tdiv) * tmulB,
// and lives in shared memory at  l * lsl + (j + (j >> psh)) * lsj  of its field's
// region (`region` elements per field).  t and y tiles keep the global order (lines contiguous: lsl = 1,
// lsj = nlines); x tiles are rows stored row by row with an odd padded row stride
// (lsj = 1, lsl = nx + 1), so every stage's accesses are bank-conflict free.
struct TileGeom {
    int nlines;
    int ntiles;
    unsigned lsl, lsj, region;
    FastDiv tdiv;
    FastDiv nl;      // nlines
    FastDiv rowlen;  // x tiles: line length nx (row-major staging)
    unsigned tmulA, tmulB;
    unsigned gs_j, gs_l;
    int pairs;       // t / y tiles: line pairs start 16-byte aligned (FP32 staging by 16 B)
    // t / y tiles: element j of a line sits at row j + (j >> psh) (one padding row of lsj
    // elements after every 2^psh rows, 2^psh the radix of the last forward stage); 31: none.
    unsigned psh = 31;
};

template <typename C> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };

// Phase-table entry: the field's own complex type (FP64 values rounded once on upload).
template <typename C> struct TabOf { using type = C; };

template <typename C> struct TPassArgs {
    using T = typename RealOf<C>::type;
    C *f[3];            // pump, signal, idler (updated in place)
    const C *psrc;      // pump source: Api when the pass starts a round trip, else f[0]
    TileGeom g;
    AxisPlan plan;
    const C *tw;        // stage twiddles of the t axis
    const typename TabOf<C>::type *tab[3];  // phase table per field (digit-reversed order)
    unsigned tmask;     // fields that get the t-axis transform
    int n_rk4;          // coupled-wave half steps before the transform (0, 1, 2)
    int use_phase;      // apply exp(-/+ i dk z) (corrected physics)
    T kappa[3];
    T c1, c3, h6;       // RK4 stage offsets (k1, k2 -> c1; k3 -> c3) and final weight h/6
    T c1k[3], c3k[3], h6k[3];  // the same times kappa of each field
    C ph[2][3];         // exp(i dk z) at the stage positions z, z+h/2, z+h of each half step
    const C *ph_steps;  // batched passes: the ph values of every t-pass of a round trip, [tp][2][3]
    int skip_rows;      // shipped quirk: transform only row y = 0 (tiles with y != 0 skip)
    unsigned nx;        // grid width (for the row test above)
    const C *eom;       // per time sample: exp(i beta sin(2 pi fpm t)) on signal and idler
                        // after the half steps (closing pass of a round trip), or null
    int line_nt;        // line-specialised FP32 form (tpass_line.cuh): its time axis, else 0
};

template <typename C> struct AxisArgs {
    C *f[3];
    TileGeom g;
    AxisPlan plan;
    const C *tw;
    const typename TabOf<C>::type *tab[3];
    unsigned tmask;
};

// Fused (x, y) diffraction pass over whole (field, t) planes.  A cluster of K CTAs owns
// one plane: CTA r first holds rows [r ny/K, (r+1) ny/K) in its slab (x geometry gx:
// rows of nx + 1 elements) and applies the x factor to them; after a cluster barrier
// it gathers columns [r nx/K, (r+1) nx/K) of every slab through distributed shared
// memory into its column region (y geometry gy: lines = columns, contiguous), applies
// the y factor and writes the columns back to global memory.
template <typename C> struct PlaneArgs {
    C *f[3];
    AxisPlan px, py;
    TileGeom gx, gy;
    FastDiv rows;       // rows per CTA (ny / K): row -> owning CTA of the cluster
    const C *twx, *twy;
    const typename TabOf<C>::type *tabx[3], *taby[3];
    unsigned tmask;     // fields transformed (one plane per field and t)
    unsigned nx, ny, nt;
    unsigned K;         // CTAs per plane (cluster size)
    unsigned regionA;   // elements of the slab region (the column region follows it)
};

// Warp-specialised passes (ws_pass.cu): a producer warp streams tiles into a ring of
// shared-memory stages with TMA (tensor copies of t / y tiles over the field viewed as a
// 3-D tensor (nx, ny, nt) of 8-byte elements, or one bulk copy per x-tile row); the
// consumer warps run the tile bodies.  Shared memory: kWsHeaderBytes of mbarriers and a
// flag, then nstages stages of stage_bytes.
constexpr unsigned kWsMaxStages = 4;
constexpr unsigned kWsHeaderBytes = 128;
constexpr unsigned kWsTabPtrOffset = 80;  // header: three phase-table pointers (after the mbarriers and flag)
enum { kWsTensor = 0, kWsRows = 1 };
struct WsArgs {
    int *err;               // error word in global memory (0: no error)
    unsigned nstages;       // ring depth (<= kWsMaxStages)
    unsigned stage_bytes;   // one stage: the three field regions (128-byte multiple)
    unsigned field_bytes;   // bytes one field's copies of a tile deliver
    int mode;               // kWsTensor / kWsRows
    // tensor mode: tile -> (tile % tdiv, tile / tdiv) = (x block, row y or plane t); the box
    // covers px pixels (inner, px * inner_mult elements) and box_lines lines along
    // line_dim (2: t for the t-pass, 1: y for the y-pass); lines / box_lines boxes per field
    unsigned px, inner_mult, line_dim, lines, box_lines;
    unsigned row_bytes;     // rows mode: bytes per row copy
    // axis passes: byte offset in dynamic shared memory where the consumers copy the stage
    // twiddles (ntw values) and the phase tables of the transformed fields (plan.n values
    // each) before the first tile; 0: the tables are read from global memory
    unsigned tab_off, ntw;
    // bound of the consumers' and the producer's ring waits in SM clock cycles (0: ~2 s);
    // the producer's final drain of its issued copies always keeps the ~2 s bound
    long long wait_cycles;
};

// Kernel variant of one pass: CTA size and first-stage radix; the largest radix any
// stage may use follows from the precision and CTA size (max_radix()).
struct PassVariant {
    int threads;  // 128 or 256; 160 or 288: warp-specialised (128 / 256 consumers + a producer warp)
    int r1;       // 4, 8 or 16, plus kLineForm for the line-specialised t-pass
};

// Flag in PassVariant::r1 (and in the r1 entries of the C-ABI tuning arrays): the
// line-specialised t-pass (tpass_line.cuh: tiles of 8 FP32 or 4 FP64 pixels, FP32
// split-pair arithmetic) on CTAs of 128 threads, for every time axis with a compiled
// body (64, 128, 256; the body fixes its own radices).  Grids it does not cover (another
// time axis, nx not a multiple of the tile, the shipped Q2 launch grid) run the generic
// tile body at the same CTA size with the fallback radix: the variant's radix in FP32,
// radix 4 (the register form) in FP64.
constexpr int kLineForm = 256;
inline int line_pixels(bool fp64) { return fp64 ? 4 : 8; }  // pixels per tile
inline bool is_line(PassVariant v) { return (v.r1 & kLineForm) != 0; }
inline int radix_of(PassVariant v) { return v.r1 & (kLineForm - 1); }
// Line-specialised t-pass kernels: CTA size and the radix of the generic fallback.
inline bool line_variant_compiled(int threads, int r1) { return threads == 128 && (r1 == 4 || r1 == 8 || r1 == 16); }
inline int line_fallback_radix(bool fp64, PassVariant v) { return fp64 ? 4 : radix_of(v); }
// First-stage radix of the compiled line body for a time axis of n samples (0: none).
inline int line_radix(int n) { return (n == 256 || n == 128) ? 16 : (n == 64 ? 8 : 0); }
// Largest radix of the generic fallback body at a line variant's CTA size.
template <typename C, int THREADS> struct LineFallback {
    static constexpr int RMAX = (sizeof(C) == 16 && THREADS == 128) ? 8 : 16;
};

inline bool is_ws(PassVariant v) { return v.threads == 160 || v.threads == 288; }
inline int consumer_threads(PassVariant v) { return is_ws(v) ? v.threads - 32 : v.threads; }
inline int max_radix(bool fp64, int threads) { return (fp64 && threads == 128) ? 8 : 16; }
// Largest radix of a variant: the warp-specialised kernels always take radix 16.
inline int variant_max_radix(bool fp64, PassVariant v) { return is_ws(v) ? 16 : max_radix(fp64, v.threads); }
bool ws_variant_compiled(bool fp64, bool tpass, PassVariant consumers);

// Whether (threads, r1) is one of the compiled variants (OPO_T_VARIANTS / OPO_A_VARIANTS
// in ssfm_kernels.cu) for the t-pass (tpass = true) or the axis passes.
inline bool variant_compiled(bool fp64, bool tpass, PassVariant v)
{
    if (is_line(v)) return tpass && line_variant_compiled(v.threads, radix_of(v));
    if (is_ws(v)) return ws_variant_compiled(fp64, tpass, PassVariant{v.threads - 32, v.r1});
    if (v.threads != 128 && v.threads != 256) return false;
    if (v.r1 != 4 && v.r1 != 8 && v.r1 != 16) return false;
    if (!fp64) return true;
    // FP64: 128-thread CTAs take radix <= 8 (registers); the t-pass's first stage holds
    // 3 fields x r1 complex128 with the RK4 state, r1 <= 8 (its split form for a radix-16
    // first stage measured slower in FP64: one dependent FP64 chain per thread)
    if (v.threads == 128 || tpass) return v.r1 <= 8;
    return true;
}

// Launchers (ssfm_kernels.cu).  smem in bytes; grid = number of CTAs.  They return
// cudaErrorInvalidValue for a variant that is not compiled.
template <typename C> cudaError_t launch_tpass(const TPassArgs<C> &a, PassVariant v, int grid, size_t smem,
                                               cudaStream_t st);
// Line-specialised t-pass (v.r1 carries kLineForm) for a time axis of nt samples; nt = 0:
// the generic tile body at the variant's CTA size with first-stage radix r_fallback
// (the plan's).
template <typename C>
cudaError_t launch_tpass_line(const TPassArgs<C> &a, PassVariant v, int nt, int r_fallback, int grid, size_t smem,
                              cudaStream_t st);
// Dynamic shared memory of a line-specialised t-pass CTA (0: nt / r1 not compiled).
size_t tpass_line_smem(bool fp64, int nt, int r1);
cudaError_t configure_line_kernels(size_t max_smem);
template <typename C> cudaError_t launch_axis(const AxisArgs<C> &a, PassVariant v, bool bfast, int grid,
                                              size_t smem, cudaStream_t st);
template <typename C> cudaError_t launch_sums(const C *f0, const C *f1, const C *f2, size_t n,
                                              double *partials, int nblocks, double *out,
                                              cudaStream_t st);
cudaError_t launch_convert_d2f(const double2 *src, float2 *dst, size_t n, cudaStream_t st);
cudaError_t launch_convert_f2d(const float2 *src, double2 *dst, size_t n, cudaStream_t st);
cudaError_t configure_kernels(size_t max_smem);
// Warp-specialised launchers (ws_pass.cu); v.threads = consumer threads (128 / 256).
// maps: tensor maps of the three fields the pass loads (t-pass: pump source, signal, idler).
cudaError_t configure_ws_kernels(size_t max_smem);
template <typename C> int ws_occupancy(bool tpass, PassVariant v, bool bfast, size_t smem);
template <typename C>
cudaError_t launch_tpass_ws(const TPassArgs<C> &a, const WsArgs &w, const CUtensorMap *maps, PassVariant v, int grid,
                            size_t smem, cudaStream_t st);
template <typename C>
cudaError_t launch_axis_ws(const AxisArgs<C> &a, const WsArgs &w, const CUtensorMap *maps, PassVariant v, bool bfast,
                           int grid, size_t smem, cudaStream_t st);

// Plane pass (plane_pass.cu).  Compiled CTA sizes: 256 and 512; the largest radix is
// plane_max_radix().  grid = planes x K CTAs in clusters of K.
inline int plane_max_radix(bool fp64) { return fp64 ? 8 : 16; }
inline bool plane_variant_compiled(int threads) { return threads == 256 || threads == 512; }
template <typename C> cudaError_t launch_plane(const PlaneArgs<C> &a, int threads, unsigned planes, size_t smem,
                                               cudaStream_t st);
// Clusters of K CTAs with `smem` bytes each that can be resident at once (0: none).
template <typename C> int plane_max_clusters(int threads, int K, size_t smem);
cudaError_t configure_plane_kernels(size_t max_smem);

}  // namespace opo
