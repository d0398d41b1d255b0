// Tile bodies of the split-step passes, shared by the single-instance kernels
// (ssfm_kernels.cu) and the batched kernels (batch.cu).
//
// Every z-step of the reference (Solver3D.cuh:946-960: RK4(dz/2), dispersion,
// diffraction, RK4(dz/2)) is executed as three passes over the resident fields, each
// reading and writing the three complex fields once:
//   t-pass    coupled-wave RK4 half steps (all stages in registers; a radix-16 first
//             stage runs them as a sweep over the staged tile first, tpass_tile_split)
//             fused with the t-axis operator: transform, times the dispersion phase,
//             inverse transform
//   x-pass,   the separable diffraction operator exp(-i dz 2 pi^2 (fx^2 + fy^2) / k)
//   y-pass    = (x factor) (y factor), one axis per pass.
// A CTA owns a tile of whole lines of one axis for all three fields, staged in shared
// memory (TileGeom gives the layout).  The first forward stage reads global memory
// directly into registers (in the t-pass it also applies the RK4 half steps), the middle
// stages exchange through shared memory, the last forward stage, the phase multiply and
// the first inverse stage are one register step, and the last inverse stage writes
// global memory directly.
//
// Index arithmetic is 32-bit (a field holds fewer than 2^32 values) and every division
// by a run-time invariant uses a precomputed multiply-high (FastDiv).  Field f of a tile
// lives in shared-memory region f.  Every body ends with the CTA synchronised.
#pragma once

#include "fft_radix.cuh"
#include "opo_internal.h"

namespace opo {

template <int S, typename C> __device__ __forceinline__ C twmul(C x, C w)
{
    // w holds exp(-2 pi i e / L); a stage of sign S multiplies by exp(S 2 pi i e / L)
    return S < 0 ? cmul(x, w) : cmulc(x, w);
}

__device__ __forceinline__ double2 tab_mul(double2 x, double2 t) { return cmul(x, t); }
__device__ __forceinline__ float2 tab_mul(float2 x, float2 t) { return cmul(x, t); }

__device__ __forceinline__ unsigned tile_base(const TileGeom &g, unsigned tile)
{
    const unsigned hi = fdiv(g.tdiv, tile);
    return (tile - hi * g.tdiv.d) * g.tmulA + hi * g.tmulB;
}

// Shared-memory row of element j of a line (padding rows included), and the row stride
// of a stage of stride q.  Every stage but the last forward one has q a multiple of
// 2^psh, so row(j0 + m q) = row(j0) + m qrow(q); the last forward stage (q = 1, radix
// 2^psh) reads row(g0 R + m) = g0 (R + 1) + m, so consecutive butterflies alternate
// between the two halves of the shared-memory banks when a line group is narrower than
// a wavefront.
__device__ __forceinline__ unsigned prow(const TileGeom &g, unsigned j) { return j + (j >> g.psh); }
__device__ __forceinline__ unsigned qrow(const TileGeom &g, unsigned q) { return q + (q >> g.psh); }

// ---------------------------------------------------------------------------------
// Tile staging with cp.async: every thread issues its share of the whole tile (all
// fields) as asynchronous global -> shared copies, so a tile costs one memory latency
// however many fields and items it has, and no registers hold the data in flight.
// Completion is the hardware wait cp.async.wait_all (no polling loop).

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
template <int BYTES> __device__ __forceinline__ void cp_async(void *dst, const void *src)
{
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Copy the raw lines of tile `tile` of the fields in mask (field f from src[f]) into their
// shared-memory regions: t / y tiles element e = j nlines + l (lines contiguous in global
// memory, two at a time when g.pairs) placed at l + prow(j) lsj, x tiles element
// e = l nx + j (rows contiguous) placed at l lsl + j.
template <typename C, int THREADS, bool ROWMAJOR>
__device__ __forceinline__ void stage_tile(const TileGeom &g, unsigned n, unsigned tile, const C *const *src,
                                           unsigned mask, C *sm)
{
    const unsigned base = tile_base(g, tile);
    const unsigned count = n * (unsigned)g.nlines;
#pragma unroll
    for (int f = 0; f < 3; f++) {
        if (!(mask & (1u << f))) continue;
        const C *gsrc = src[f] + base;
        C *dst = sm + (size_t)f * g.region;
        if (ROWMAJOR) {
            for (unsigned e = threadIdx.x; e < count; e += THREADS) {
                const unsigned l = fdiv(g.rowlen, e), j = e - l * n;
                cp_async<sizeof(C)>(dst + l * g.lsl + j, gsrc + e);
            }
        } else if (sizeof(C) == 8 && g.pairs) {
            for (unsigned e = 2 * threadIdx.x; e < count; e += 2 * THREADS) {
                const unsigned j = fdiv(g.nl, e), l = e - j * g.nlines;
                cp_async<16>(dst + l + prow(g, j) * g.lsj, gsrc + j * g.gs_j + l);
            }
        } else {
            for (unsigned e = threadIdx.x; e < count; e += THREADS) {
                const unsigned j = fdiv(g.nl, e), l = e - j * g.nlines;
                cp_async<sizeof(C)>(dst + l + prow(g, j) * g.lsj, gsrc + j * g.gs_j + l);
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

// CTA-wide barrier of a tile body: BAR = 0 is __syncthreads(); BAR > 0 is named
// barrier 1 over the first BAR threads (the consumer warps of a warp-specialised CTA,
// whose producer warp never joins it).
template <int BAR> __device__ __forceinline__ void tile_sync()
{
    if constexpr (BAR == 0)
        __syncthreads();
    else
        asm volatile("bar.sync 1, %0;\n" ::"n"(BAR) : "memory");
}

// Index of the f-th field (in p, s, i order) selected by mask.
__device__ __forceinline__ int field_id(unsigned mask, int f)
{
    // the f-th set bit of a three-bit mask, without branches: clear the lowest set bit f times
    mask = f > 0 ? mask & (mask - 1) : mask;
    mask = f > 1 ? mask & (mask - 1) : mask;
    return __ffs(mask) - 1;
}

// ---------------------------------------------------------------------------------
// Shared-memory stages.  Per field, work item w -> (line l fastest, butterfly b).
//
// The stage functions take WS = true in the warp-specialised kernels (consumer warps of
// a CTA with a producer warp).  Two things follow from it:
//  * for_items runs body(w, fields) over every item of every field in mask.  A thread
//    takes whole items and runs all their fields (the index arithmetic of an item is done
//    once).  With WS, whose 128 / 256 consumer threads often outnumber a stage's items,
//    when that would not load every thread evenly -- the most butterflies one thread
//    runs, nf * ceil(items / THREADS), exceeds ceil(nf * items / THREADS) -- the
//    (field, item) pairs are spread over the threads instead.  The other kernels compile
//    the first form only: the second, even unused, costs them 3-7 %.
//  * ldtab<WS> reads twiddles and phase tables: __ldg from global memory, or with WS a
//    generic load, since those kernels may hold the tables in shared memory.
template <bool WS, typename T> __device__ __forceinline__ T ldtab(const T *p)
{
    if constexpr (WS)
        return *p;
    else
        return __ldg(p);
}

template <int THREADS, bool WS, typename F>
__device__ __forceinline__ void for_items(unsigned items, unsigned mask, F &&body)
{
    const unsigned nf = __popc(mask);
    if (!WS || nf * ((items + THREADS - 1) / THREADS) <= (nf * items + THREADS - 1) / THREADS) {
        for (unsigned w = threadIdx.x; w < items; w += THREADS) body(w, mask);
    } else if constexpr (WS) {
        for (unsigned u = threadIdx.x; u < nf * items; u += THREADS) {
            const unsigned fi = (u >= items) + (u >= 2 * items);
            body(u - fi * items, 1u << field_id(mask, (int)fi));
        }
    }
}

template <typename C, int R, int S, bool DIT, int THREADS, bool WS = false>
__device__ void smem_stage(C *sm, const TileGeom &g, int n, int L, const FastDiv &fq, const C *tw, unsigned mask)
{
    // per item: the index arithmetic once, then every field in mask
    const unsigned q = fq.d, nl = (unsigned)g.nlines, lsl = g.lsl, lsj = g.lsj, qs = qrow(g, q) * lsj;
    const unsigned items = (unsigned)(n / R) * nl;
    for_items<THREADS, WS>(items, mask, [&](unsigned w, unsigned fm) {
        const unsigned b = fdiv(g.nl, w), l = w - b * nl;
        const unsigned gq = fdiv(fq, b), j = b - gq * q;
        const unsigned off = l * lsl + prow(g, gq * L + j) * lsj;
        const C *tj = tw + j;
        for (unsigned fb = fm; fb; fb &= fb - 1) {
            const int f = __ffs(fb) - 1;
            C *sp = sm + (size_t)f * g.region + off;
            C x[R];
#pragma unroll
            for (int m = 0; m < R; m++) x[m] = sp[m * qs];
            if (DIT && q > 1) {
#pragma unroll
                for (int m = 1; m < R; m++) x[m] = twmul<S>(x[m], ldtab<WS>(tj + (m - 1) * q));
            }
            dft<R, S>(x);
            if (!DIT && q > 1) {
#pragma unroll
                for (int k = 1; k < R; k++) x[k] = twmul<S>(x[k], ldtab<WS>(tj + (k - 1) * q));
            }
#pragma unroll
            for (int k = 0; k < R; k++) sp[k * qs] = x[k];
        }
    });
}

// Last forward stage (q = 1), phase multiply, first inverse stage, in registers.
template <typename C, int R, int SF, int THREADS, bool WS = false>
__device__ void fused_middle(C *sm, const TileGeom &g, int n, const typename TabOf<C>::type *const *tab,
                             unsigned mask)
{
    const unsigned nl = (unsigned)g.nlines, lsl = g.lsl, lsj = g.lsj;
    const unsigned items = (unsigned)(n / R) * nl;
    for_items<THREADS, WS>(items, mask, [&](unsigned w, unsigned fm) {
        const unsigned g0 = fdiv(g.nl, w), l = w - g0 * nl;
        const unsigned off = l * lsl + g0 * qrow(g, R) * lsj;
        for (unsigned fb = fm; fb; fb &= fb - 1) {
            const int f = __ffs(fb) - 1;
            C *sp = sm + (size_t)f * g.region + off;
            const typename TabOf<C>::type *tb = tab[f] + g0 * R;
            C x[R];
#pragma unroll
            for (int m = 0; m < R; m++) x[m] = sp[m * lsj];
            dft<R, SF>(x);
#pragma unroll
            for (int k = 0; k < R; k++) x[k] = tab_mul(x[k], ldtab<WS>(tb + k));
            dft<R, -SF>(x);
#pragma unroll
            for (int k = 0; k < R; k++) sp[k * lsj] = x[k];
        }
    });
}

template <typename C, int S, bool DIT, int THREADS, int RMAX, bool WS = false>
__device__ void smem_stage_dispatch(int R, C *sm, const TileGeom &g, int n, int L, const FastDiv &fq,
                                    const C *tw, unsigned mask)
{
    switch (R) {
    case 2: smem_stage<C, 2, S, DIT, THREADS, WS>(sm, g, n, L, fq, tw, mask); break;
    case 3: smem_stage<C, 3, S, DIT, THREADS, WS>(sm, g, n, L, fq, tw, mask); break;
    case 4: smem_stage<C, 4, S, DIT, THREADS, WS>(sm, g, n, L, fq, tw, mask); break;
    case 8: smem_stage<C, 8, S, DIT, THREADS, WS>(sm, g, n, L, fq, tw, mask); break;
    case 16:
        if constexpr (RMAX >= 16) smem_stage<C, 16, S, DIT, THREADS, WS>(sm, g, n, L, fq, tw, mask);
        break;
    default: break;
    }
}

template <typename C, int SF, int THREADS, int RMAX, bool WS = false>
__device__ void fused_dispatch(int R, C *sm, const TileGeom &g, int n, const typename TabOf<C>::type *const *tab,
                               unsigned mask)
{
    switch (R) {
    case 2: fused_middle<C, 2, SF, THREADS, WS>(sm, g, n, tab, mask); break;
    case 3: fused_middle<C, 3, SF, THREADS, WS>(sm, g, n, tab, mask); break;
    case 4: fused_middle<C, 4, SF, THREADS, WS>(sm, g, n, tab, mask); break;
    case 8: fused_middle<C, 8, SF, THREADS, WS>(sm, g, n, tab, mask); break;
    case 16:
        if constexpr (RMAX >= 16) fused_middle<C, 16, SF, THREADS, WS>(sm, g, n, tab, mask);
        break;
    default: break;
    }
}

// Stages 1 .. ns-1 forward, fused middle, inverse back to stage 1 (stage 0 is fused
// with the global load / store by the caller).
template <typename C, int SF, int THREADS, int RMAX, int BAR = 0>
__device__ __forceinline__ void middle_stages(C *sm, const TileGeom &g, const AxisPlan &p, const C *tw,
                              const typename TabOf<C>::type *const *tab, unsigned mask)
{
    for (int s = 1; s < p.ns - 1; s++) {
        smem_stage_dispatch<C, SF, false, THREADS, RMAX, (BAR > 0)>(p.radix[s], sm, g, p.n, p.len[s], p.q[s],
                                                         tw + p.twoff[s], mask);
        tile_sync<BAR>();
    }
    fused_dispatch<C, SF, THREADS, RMAX, (BAR > 0)>(p.radix[p.ns - 1], sm, g, p.n, tab, mask);
    tile_sync<BAR>();
    for (int s = p.ns - 2; s >= 1; s--) {
        smem_stage_dispatch<C, -SF, true, THREADS, RMAX, (BAR > 0)>(p.radix[s], sm, g, p.n, p.len[s], p.q[s],
                                                         tw + p.twoff[s], mask);
        tile_sync<BAR>();
    }
}

// Last inverse stage (radix R1, stride q) of every field in mask, written to global:
// per item the index arithmetic once, then each field.
template <typename C, int R1, int SB, bool BFAST, int THREADS, bool WS = false>
__device__ __forceinline__ void final_stage(C *sm, const TileGeom &g, unsigned n, unsigned base, C *const *dst,
                                            const C *tw, const FastDiv &fq0, unsigned mask)
{
    const unsigned q = n / R1, nl = (unsigned)g.nlines, items = q * nl, qs = qrow(g, q) * g.lsj;
    for_items<THREADS, WS>(items, mask, [&](unsigned w, unsigned fm) {
        unsigned b, l;
        if (BFAST) {
            l = fdiv(fq0, w);
            b = w - l * q;
        } else {
            b = fdiv(g.nl, w);
            l = w - b * nl;
        }
        const unsigned soff = l * g.lsl + prow(g, b) * g.lsj, goff = base + l * g.gs_l + b * g.gs_j;
        const C *tb = tw + b;
        for (unsigned fb = fm; fb; fb &= fb - 1) {
            const int f = __ffs(fb) - 1;
            const C *sp = sm + (size_t)f * g.region + soff;
            C x[R1];
#pragma unroll
            for (int m = 0; m < R1; m++) x[m] = sp[m * qs];
#pragma unroll
            for (int m = 1; m < R1; m++) x[m] = twmul<SB>(x[m], ldtab<WS>(tb + (m - 1) * q));
            dft<R1, SB>(x);
            C *d = dst[f] + goff;
#pragma unroll
            for (int k = 0; k < R1; k++) d[k * q * g.gs_j] = x[k];
        }
    });
}

// ---------------------------------------------------------------------------------
// Coupled-wave equations, reference Solver3D.cuh:365-425 and :872-943.
//   dAp = i kp As Ai e^{-i dk z}, dAs = i ks Ap Ai* e^{i dk z}, dAi = i ki Ap As* e^{i dk z}
// One half step of size h = dz/2: k1 = f(A), k2 = f(A + c1 k1), k3 = f(A + c1 k2),
// k4 = f(A + c3 k3), A += (k1 + 2 k2 + 2 k3 + k4) h / 6.  The shipped stage offsets are
// c1 = 0.5, c3 = 1 (no step size); corrected physics uses c1 = h/2, c3 = h.

template <typename C, typename T>
__device__ __forceinline__ void cwe_rhs(const T *kap, C p, C s, C i, C &dp, C &ds, C &di)
{
    C si = cmul(s, i), pic = cmulc(p, i), psc = cmulc(p, s);
    dp = C{-kap[0] * si.y, kap[0] * si.x};
    ds = C{-kap[1] * pic.y, kap[1] * pic.x};
    di = C{-kap[2] * psc.y, kap[2] * psc.x};
}

template <typename C, typename T>
__device__ __forceinline__ void cwe_rhs_phase(const T *kap, const C &ph, C p, C s, C i, C &dp, C &ds,
                                              C &di)
{
    cwe_rhs(kap, p, s, i, dp, ds, di);
    dp = cmulc(dp, ph);
    ds = cmul(ds, ph);
    di = cmul(di, ph);
}

// The products u_p = s i, u_s = p i*, u_i = p s* give k = i kappa u, so every use of k
// (the next stage's A + c k and the final sum) folds kappa and the step weights into
// precomputed constants: A + c k = (A.x - c kappa u.y, A.y + c kappa u.x), and
// A += (h/6) kappa i (u1 + 2 u2 + 2 u3 + u4).  The products and their weighted sum are
// held with their components swapped, w = (u.y, u.x), so that A + c k = A + (-c kappa,
// c kappa) * w componentwise: one packed f32x2 fused multiply-add in FP32.
template <typename C> __device__ __forceinline__ C swp(C u) { return C{u.y, u.x}; }
template <typename C, typename T>
__device__ __forceinline__ C add_iku_w(C a, T ck, C w)
{
    return C{a.x - ck * w.x, a.y + ck * w.y};
}
template <> __device__ __forceinline__ float2 add_iku_w<float2, float>(float2 a, float ck, float2 w)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2pack(float2{-ck, ck})), "l"(f2pack(w)), "l"(f2pack(a)));
    return f2unpack(d);
}

template <typename C>
__device__ __forceinline__ void rk4_half_fast(const TPassArgs<C> &a, C &p, C &s, C &i)
{
    using T = typename TPassArgs<C>::T;
    C up = swp(cmul(s, i)), us = swp(cmulc(p, i)), ui = swp(cmulc(p, s));  // stage 1
    C Up = up, Us = us, Ui = ui;
    C p2 = add_iku_w(p, a.c1k[0], up), s2 = add_iku_w(s, a.c1k[1], us), i2 = add_iku_w(i, a.c1k[2], ui);
    up = swp(cmul(s2, i2)); us = swp(cmulc(p2, i2)); ui = swp(cmulc(p2, s2));  // stage 2
    Up = caxpy(T(2), up, Up);
    Us = caxpy(T(2), us, Us);
    Ui = caxpy(T(2), ui, Ui);
    p2 = add_iku_w(p, a.c1k[0], up); s2 = add_iku_w(s, a.c1k[1], us); i2 = add_iku_w(i, a.c1k[2], ui);
    up = swp(cmul(s2, i2)); us = swp(cmulc(p2, i2)); ui = swp(cmulc(p2, s2));  // stage 3
    Up = caxpy(T(2), up, Up);
    Us = caxpy(T(2), us, Us);
    Ui = caxpy(T(2), ui, Ui);
    p2 = add_iku_w(p, a.c3k[0], up); s2 = add_iku_w(s, a.c3k[1], us); i2 = add_iku_w(i, a.c3k[2], ui);
    up = swp(cmul(s2, i2)); us = swp(cmulc(p2, i2)); ui = swp(cmulc(p2, s2));  // stage 4
    Up = cadd(Up, up);
    Us = cadd(Us, us);
    Ui = cadd(Ui, ui);
    p = add_iku_w(p, a.h6k[0], Up);
    s = add_iku_w(s, a.h6k[1], Us);
    i = add_iku_w(i, a.h6k[2], Ui);
}

// The same half step for two voxels at once in FP32, their real parts and imaginary parts
// each held as one packed f32x2 pair (v[0] = {re of voxel 0, re of voxel 1}, v[1] = the
// imaginary parts): every product and update then serves both voxels with one packed
// instruction per component, and a complex product costs 5 instead of 8 instructions
// for the pair.  u = s i, p i*, p s*;  A + c i kappa u  and  A += (h/6) i kappa (u1 + 2 u2 +
// 2 u3 + u4)  as in rk4_half_fast.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 x2_mul(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("mul.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 x2_add(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("add.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 x2_sub(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("sub.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 x2_fma(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f32x2 x2_dup(float s) { return f2pack(float2{s, s}); }
// a b (conj_b: a conj(b)) for pairs of complex values in split re / im form
template <bool CONJ_B>
__device__ __forceinline__ void x2_cmul(const f32x2 *a, const f32x2 *b, f32x2 *d)
{
    if (CONJ_B) {
        d[0] = x2_fma(a[0], b[0], x2_mul(a[1], b[1]));
        d[1] = x2_sub(x2_mul(a[1], b[0]), x2_mul(a[0], b[1]));
    } else {
        d[0] = x2_sub(x2_mul(a[0], b[0]), x2_mul(a[1], b[1]));
        d[1] = x2_fma(a[0], b[1], x2_mul(a[1], b[0]));
    }
}
// d = a + i c u  (c = {c, c}, nc = {-c, -c})
__device__ __forceinline__ void x2_add_iku(const f32x2 *a, f32x2 c, f32x2 nc, const f32x2 *u, f32x2 *d)
{
    d[0] = x2_fma(u[1], nc, a[0]);
    d[1] = x2_fma(u[0], c, a[1]);
}

__device__ __forceinline__ void rk4_half_fast_x2(const TPassArgs<float2> &a, f32x2 (&p)[2], f32x2 (&s)[2],
                                                 f32x2 (&i)[2])
{
    const f32x2 two = x2_dup(2.f);
    f32x2 up[2], us[2], ui[2], Up[2], Us[2], Ui[2], p2[2], s2[2], i2[2];
    x2_cmul<false>(s, i, up);
    x2_cmul<true>(p, i, us);
    x2_cmul<true>(p, s, ui);
#pragma unroll
    for (int c = 0; c < 2; c++) { Up[c] = up[c]; Us[c] = us[c]; Ui[c] = ui[c]; }
#pragma unroll
    for (int st = 1; st < 4; st++) {
        const float *ck = st < 3 ? a.c1k : a.c3k;
        x2_add_iku(p, x2_dup(ck[0]), x2_dup(-ck[0]), up, p2);
        x2_add_iku(s, x2_dup(ck[1]), x2_dup(-ck[1]), us, s2);
        x2_add_iku(i, x2_dup(ck[2]), x2_dup(-ck[2]), ui, i2);
        x2_cmul<false>(s2, i2, up);
        x2_cmul<true>(p2, i2, us);
        x2_cmul<true>(p2, s2, ui);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            if (st < 3) {
                Up[c] = x2_fma(up[c], two, Up[c]);
                Us[c] = x2_fma(us[c], two, Us[c]);
                Ui[c] = x2_fma(ui[c], two, Ui[c]);
            } else {
                Up[c] = x2_add(Up[c], up[c]);
                Us[c] = x2_add(Us[c], us[c]);
                Ui[c] = x2_add(Ui[c], ui[c]);
            }
        }
    }
    f32x2 t[2];
    x2_add_iku(p, x2_dup(a.h6k[0]), x2_dup(-a.h6k[0]), Up, t);
    p[0] = t[0]; p[1] = t[1];
    x2_add_iku(s, x2_dup(a.h6k[1]), x2_dup(-a.h6k[1]), Us, t);
    s[0] = t[0]; s[1] = t[1];
    x2_add_iku(i, x2_dup(a.h6k[2]), x2_dup(-a.h6k[2]), Ui, t);
    i[0] = t[0]; i[1] = t[1];
}

template <typename C>
__device__ __forceinline__ void rk4_half(const TPassArgs<C> &a, int h, C &p, C &s, C &i)
{
    using T = typename TPassArgs<C>::T;
    if (!a.use_phase) {
        rk4_half_fast(a, p, s, i);
        return;
    }
    C k1p, k1s, k1i, k2p, k2s, k2i, k3p, k3s, k3i, k4p, k4s, k4i;
    const T c1 = a.c1, c3 = a.c3;
    const C *ph = a.ph[h];
    cwe_rhs_phase(a.kappa, ph[0], p, s, i, k1p, k1s, k1i);
    cwe_rhs_phase(a.kappa, ph[1], C{p.x + c1 * k1p.x, p.y + c1 * k1p.y}, C{s.x + c1 * k1s.x, s.y + c1 * k1s.y},
                  C{i.x + c1 * k1i.x, i.y + c1 * k1i.y}, k2p, k2s, k2i);
    cwe_rhs_phase(a.kappa, ph[1], C{p.x + c1 * k2p.x, p.y + c1 * k2p.y}, C{s.x + c1 * k2s.x, s.y + c1 * k2s.y},
                  C{i.x + c1 * k2i.x, i.y + c1 * k2i.y}, k3p, k3s, k3i);
    cwe_rhs_phase(a.kappa, ph[2], C{p.x + c3 * k3p.x, p.y + c3 * k3p.y}, C{s.x + c3 * k3s.x, s.y + c3 * k3s.y},
                  C{i.x + c3 * k3i.x, i.y + c3 * k3i.y}, k4p, k4s, k4i);
    const T w = a.h6;
    p.x += (k1p.x + T(2) * k2p.x + T(2) * k3p.x + k4p.x) * w;
    p.y += (k1p.y + T(2) * k2p.y + T(2) * k3p.y + k4p.y) * w;
    s.x += (k1s.x + T(2) * k2s.x + T(2) * k3s.x + k4s.x) * w;
    s.y += (k1s.y + T(2) * k2s.y + T(2) * k3s.y + k4s.y) * w;
    i.x += (k1i.x + T(2) * k2i.x + T(2) * k3i.x + k4i.x) * w;
    i.y += (k1i.y + T(2) * k2i.y + T(2) * k3i.y + k4i.y) * w;
}

// Fields a t-pass must read and write: all three when it applies coupled-wave half
// steps, else the transformed ones plus the pump when it is reset from its source.
template <typename C> __device__ __forceinline__ unsigned tpass_load_mask(const TPassArgs<C> &a)
{
    return a.n_rk4 ? 7u : (a.tmask | (a.psrc != a.f[0] ? 1u : 0u));
}

// ---------------------------------------------------------------------------------
// t-pass: tile = P consecutive pixels (x) of one row y, all t, all three fields.
// Stage 0 (radix R1, stride q = nt/R1): each thread takes R1 time samples of one pixel
// for p, s, i from global memory (only the fields it changes: tpass_load_mask), applies
// n_rk4 half steps to each voxel, then the first forward stage of every transformed
// field into its shared-memory region (untransformed fields go back to global).

// Split form of the t-pass for a staged tile and a radix-16 first stage (256 = 16 x 16:
// the first stage, the fused middle and the last stage -- three register passes over the
// tile instead of five for radix 8 x 8 x 4).  Sixteen samples of three fields and the RK4
// state would not fit in registers together, so the coupled-wave half steps (and the EOM)
// run first as their own sweep over the staged tile, one voxel per thread and item, in
// place; then the first forward stage runs per field from shared memory like any other
// stage.  The FP32 variants take it (two pixels per item on packed pairs); in FP64 the
// per-thread dependent chain of a one-voxel sweep measured slower than the register
// form, so FP64 first stages stay at radix <= 8.
template <typename C, int R1, int THREADS, int RMAX, int BAR = 0>
__device__ __forceinline__ void tpass_tile_split(const TPassArgs<C> &a, unsigned tile, C *sm)
{
    const AxisPlan &p = a.plan;
    const TileGeom &g = a.g;
    const unsigned n = p.n, P = g.nlines, lsj = g.lsj;
    const unsigned base = tile_base(g, tile);
    bool xform = a.tmask != 0;
    if (a.skip_rows && base >= a.nx) xform = false;  // row y = base / nx != 0
    const unsigned tmask = xform ? a.tmask : 0u;
    const unsigned lmask = tpass_load_mask(a);
    bool swept = false;
    if constexpr (sizeof(C) == 8) {
        // FP32: two neighbouring pixels (l, l + 1) per item, their values as packed pairs
        // (16-byte shared-memory accesses; one packed instruction per component for both)
        if (g.pairs && !a.use_phase && (a.n_rk4 > 0 || a.eom || (lmask & ~tmask))) {
            for (unsigned e = 2 * threadIdx.x; e < n * P; e += 2 * THREADS) {
                const unsigned j = fdiv(g.nl, e), l = e - j * P;  // time sample j, pixels l, l + 1
                const unsigned off = l + prow(g, j) * lsj;
                f32x2 v[3][2];
#pragma unroll
                for (int f = 0; f < 3; f++) {
                    float4 q4 = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (lmask & (1u << f)) q4 = *reinterpret_cast<const float4 *>(sm + (size_t)f * g.region + off);
                    v[f][0] = f2pack(float2{q4.x, q4.z});
                    v[f][1] = f2pack(float2{q4.y, q4.w});
                }
                for (int h = 0; h < a.n_rk4; h++)
                    rk4_half_fast_x2(reinterpret_cast<const TPassArgs<float2> &>(a), v[0], v[1], v[2]);
                if (a.eom) {
                    const C ev = __ldg(a.eom + j);
                    const f32x2 er = x2_dup(ev.x), ei = x2_dup(ev.y);
                    for (int f = 1; f < 3; f++) {
                        const f32x2 re = x2_sub(x2_mul(v[f][0], er), x2_mul(v[f][1], ei));
                        v[f][1] = x2_fma(v[f][0], ei, x2_mul(v[f][1], er));
                        v[f][0] = re;
                    }
                }
                const unsigned gb = base + l * g.gs_l + j * g.gs_j;
#pragma unroll
                for (int f = 0; f < 3; f++) {
                    const float2 re = f2unpack(v[f][0]), im = f2unpack(v[f][1]);
                    const float4 q4 = make_float4(re.x, im.x, re.y, im.y);
                    if (tmask & (1u << f))
                        *reinterpret_cast<float4 *>(sm + (size_t)f * g.region + off) = q4;
                    else if (lmask & (1u << f))
                        *reinterpret_cast<float4 *>(a.f[f] + gb) = q4;
                }
            }
            tile_sync<BAR>();
            swept = true;
        }
    }
    if (!swept && (a.n_rk4 > 0 || a.eom || (lmask & ~tmask))) {
        for (unsigned e = threadIdx.x; e < n * P; e += THREADS) {
            const unsigned j = fdiv(g.nl, e), l = e - j * P;  // time sample j of pixel l
            const unsigned off = l + prow(g, j) * lsj;
            C v[3];
#pragma unroll
            for (int f = 0; f < 3; f++) v[f] = (lmask & (1u << f)) ? sm[(size_t)f * g.region + off] : C{};
            for (int h = 0; h < a.n_rk4; h++) rk4_half(a, h, v[0], v[1], v[2]);
            if (a.eom) {
                const C ev = __ldg(a.eom + j);
                v[1] = cmul(v[1], ev);
                v[2] = cmul(v[2], ev);
            }
            const unsigned gb = base + l * g.gs_l + j * g.gs_j;
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (tmask & (1u << f))
                    sm[(size_t)f * g.region + off] = v[f];
                else if (lmask & (1u << f))
                    a.f[f][gb] = v[f];
            }
        }
        tile_sync<BAR>();
    }
    if (!tmask) return;
    smem_stage_dispatch<C, +1, false, THREADS, RMAX, (BAR > 0)>(p.radix[0], sm, g, (int)n, p.len[0], p.q[0], a.tw,
                                                               tmask);
    tile_sync<BAR>();
    middle_stages<C, +1, THREADS, RMAX, BAR>(sm, g, p, a.tw, a.tab, tmask);
    final_stage<C, R1, -1, false, THREADS, (BAR > 0)>(sm, g, n, base, a.f, a.tw, p.q[0], tmask);
    tile_sync<BAR>();
}

template <typename C, int R1, int THREADS, int RMAX, bool STAGED = false, int BAR = 0>
__device__ __forceinline__ void tpass_tile(const TPassArgs<C> &a, unsigned tile, C *sm)
{
    if constexpr (STAGED && R1 >= 16) {
        tpass_tile_split<C, R1, THREADS, RMAX, BAR>(a, tile, sm);
        return;
    }
    const AxisPlan &p = a.plan;
    const TileGeom &g = a.g;
    const unsigned n = p.n, q = n / R1, P = g.nlines, lsj = g.lsj, qs = qrow(g, q) * lsj;
    const unsigned base = tile_base(g, tile);
    bool xform = a.tmask != 0;
    if (a.skip_rows && base >= a.nx) xform = false;  // row y = base / nx != 0
    const unsigned tmask = xform ? a.tmask : 0u;
    const unsigned lmask = tpass_load_mask(a);
    for (unsigned w = threadIdx.x; w < q * P; w += THREADS) {
        const unsigned b = fdiv(g.nl, w), l = w - b * P;
        const unsigned gb = base + l * g.gs_l + b * g.gs_j;
        const unsigned gstep = q * g.gs_j;
        C x[3][R1];
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (!(lmask & (1u << f))) continue;
            const C *gsrc = f == 0 ? a.psrc : a.f[f];
#pragma unroll
            for (int m = 0; m < R1; m++)
                x[f][m] = STAGED ? sm[f * g.region + l + prow(g, b) * lsj + m * qs] : gsrc[gb + m * gstep];
        }
        for (int h = 0; h < a.n_rk4; h++) {
#pragma unroll
            for (int m = 0; m < R1; m++) rk4_half(a, h, x[0][m], x[1][m], x[2][m]);
        }
        if (a.eom) {
#pragma unroll
            for (int m = 0; m < R1; m++) {
                const C e = __ldg(a.eom + b + m * q);
                x[1][m] = cmul(x[1][m], e);
                x[2][m] = cmul(x[2][m], e);
            }
        }
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (tmask & (1u << f)) {
                dft<R1, +1>(x[f]);
#pragma unroll
                for (int k = 1; k < R1; k++) x[f][k] = twmul<+1>(x[f][k], ldtab<(BAR > 0)>(a.tw + (k - 1) * q + b));
                C *s = sm + (size_t)f * g.region + l + prow(g, b) * lsj;
#pragma unroll
                for (int k = 0; k < R1; k++) s[k * qs] = x[f][k];
            } else if (lmask & (1u << f)) {
#pragma unroll
                for (int m = 0; m < R1; m++) a.f[f][gb + m * gstep] = x[f][m];
            }
        }
    }
    tile_sync<BAR>();
    if (!tmask) return;
    middle_stages<C, +1, THREADS, RMAX, BAR>(sm, g, p, a.tw, a.tab, tmask);
    final_stage<C, R1, -1, false, THREADS, (BAR > 0)>(sm, g, n, base, a.f, a.tw, p.q[0], tmask);
    tile_sync<BAR>();
}

// ---------------------------------------------------------------------------------
// Axis pass (x or y diffraction factor): forward transform sign -1 (the reference's
// CUFFT_FORWARD), phase, inverse sign +1.  BFAST maps consecutive threads to
// consecutive butterflies of a line (x axis, where lines are rows and the transform
// index is the contiguous one); otherwise consecutive threads take consecutive lines.

template <typename C, int R1, bool BFAST, int THREADS, int RMAX, bool STAGED = false, int BAR = 0>
__device__ __forceinline__ void axis_tile(const AxisArgs<C> &a, unsigned tile, C *sm, const C *tw,
                                          const typename TabOf<C>::type *const *tab)
{
    const AxisPlan &p = a.plan;
    const TileGeom &g = a.g;
    const unsigned n = p.n, q = n / R1, NL = g.nlines, qs = qrow(g, q) * g.lsj;
    const int nf = __popc(a.tmask);
    const unsigned items = q * NL;
    if (nf == 0) {
        tile_sync<BAR>();
        return;
    }
    const unsigned base = tile_base(g, tile);
    if constexpr (!STAGED && sizeof(C) == 8 && R1 <= 8) {
        // FP32 first stage from global memory: every field's values of an item are loaded
        // before any is transformed, three times the loads in flight per thread
        for (unsigned w = threadIdx.x; w < items; w += THREADS) {
            unsigned b, l;
            if (BFAST) {
                l = fdiv(p.q[0], w);
                b = w - l * q;
            } else {
                b = fdiv(g.nl, w);
                l = w - b * NL;
            }
            const unsigned gb = base + l * g.gs_l + b * g.gs_j, off = l * g.lsl + prow(g, b) * g.lsj;
            C x[3][R1];
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (!(a.tmask & (1u << f))) continue;
#pragma unroll
                for (int m = 0; m < R1; m++) x[f][m] = a.f[f][gb + m * q * g.gs_j];
            }
#pragma unroll
            for (int f = 0; f < 3; f++) {
                if (!(a.tmask & (1u << f))) continue;
                dft<R1, -1>(x[f]);
#pragma unroll
                for (int k = 1; k < R1; k++) x[f][k] = twmul<-1>(x[f][k], ldtab<false>(tw + (k - 1) * q + b));
                C *sp = sm + (size_t)f * g.region + off;
#pragma unroll
                for (int k = 0; k < R1; k++) sp[k * qs] = x[f][k];
            }
        }
    } else
    for (int f = 0; f < nf; f++) {
        const int fid = field_id(a.tmask, f);
        const C *srcf = a.f[fid] + base;
        C *sf = sm + (size_t)fid * g.region;
        for (unsigned w = threadIdx.x; w < items; w += THREADS) {
            unsigned b, l;
            if (BFAST) {
                l = fdiv(p.q[0], w);
                b = w - l * q;
            } else {
                b = fdiv(g.nl, w);
                l = w - b * NL;
            }
            C *s = sf + l * g.lsl + prow(g, b) * g.lsj;
            C x[R1];
#pragma unroll
            for (int m = 0; m < R1; m++) x[m] = STAGED ? s[m * qs] : srcf[l * g.gs_l + (b + m * q) * g.gs_j];
            dft<R1, -1>(x);
#pragma unroll
            for (int k = 1; k < R1; k++) x[k] = twmul<-1>(x[k], ldtab<(BAR > 0)>(tw + (k - 1) * q + b));
#pragma unroll
            for (int k = 0; k < R1; k++) s[k * qs] = x[k];
        }
    }
    tile_sync<BAR>();
    middle_stages<C, -1, THREADS, RMAX, BAR>(sm, g, p, tw, tab, a.tmask);
    final_stage<C, R1, +1, BFAST, THREADS, (BAR > 0)>(sm, g, n, base, a.f, tw, p.q[0], a.tmask);
    tile_sync<BAR>();
}

// The same with the pass's own twiddle and phase-table pointers.
template <typename C, int R1, bool BFAST, int THREADS, int RMAX, bool STAGED = false, int BAR = 0>
__device__ __forceinline__ void axis_tile(const AxisArgs<C> &a, unsigned tile, C *sm)
{
    axis_tile<C, R1, BFAST, THREADS, RMAX, STAGED, BAR>(a, tile, sm, a.tw, a.tab);
}

}  // namespace opo
