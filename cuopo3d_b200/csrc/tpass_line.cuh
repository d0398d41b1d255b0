// Line-specialised FP32 t-pass: the tile body of tpass_tile / tpass_tile_split for a
// time axis whose length and radix plan are compile-time constants (NT = RA x RB with
// RA, RB in {8, 16}: 64, 128, 256) and a tile of P = 8 pixels of one row.
//
// It computes what the split t-pass computes (reference Solver3D.cuh:872-943 RK4 half
// steps, then Solver3D.cuh:572-639 dispersion: transform, phase, inverse transform),
// with three changes of form:
//  * every value is held as a split pair: the same time sample of pixels l and l + 1,
//    real parts in one packed f32x2 register pair and imaginary parts in another, both in
//    registers and in shared memory (16 bytes: re_l, re_l+1, im_l, im_l+1).  Every
//    butterfly, twiddle and phase product then serves two lines with one packed
//    instruction per component: a complex product costs 4 packed instructions for two
//    values instead of 4 scalar ones for one, and multiplying by +-i only renames
//    registers;
//  * each twiddle and phase factor is loaded once for both lines and duplicated into
//    both lanes of a pair;
//  * all index arithmetic is compile-time: the tile, the rows and the butterfly of an
//    item follow from shifts and masks.
// The transforms are the generic two-stage plan [RA, RB] (decimation in frequency
// forward, in time inverse, phase tables in the plan's digit-reversed order), so the
// twiddles and phase tables are the host's tables of that plan.
//
// Shared memory per field: (NT + NT / RB) rows of P / 2 split pairs; time sample t sits
// in row t + t / RB (a padding row after every RB rows), so the RB-point stage's eight
// butterflies of a warp fall on alternating halves of the banks, and the other stages
// read whole 512-byte runs.
#pragma once

#include "pass_body.cuh"

namespace opo {

struct X2C {
    f32x2 r, i;
};

// Packed FP32 arithmetic with explicit rounding (no contraction left to the compiler):
// the single-instance and batched kernels that share this body compute bit-identical
// results.
__device__ __forceinline__ f32x2 xr_add(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 xr_sub(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 xr_mul(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 xr_fma(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__device__ __forceinline__ X2C xadd(X2C a, X2C b) { return X2C{xr_add(a.r, b.r), xr_add(a.i, b.i)}; }
__device__ __forceinline__ X2C xsub(X2C a, X2C b) { return X2C{xr_sub(a.r, b.r), xr_sub(a.i, b.i)}; }
// a (c + i s) and a (c - i s); ns = -s
__device__ __forceinline__ X2C xmul(X2C a, f32x2 c, f32x2 s, f32x2 ns)
{
    return X2C{xr_fma(a.i, ns, xr_mul(a.r, c)), xr_fma(a.r, s, xr_mul(a.i, c))};
}
__device__ __forceinline__ X2C xmulc(X2C a, f32x2 c, f32x2 s, f32x2 ns)
{
    return X2C{xr_fma(a.i, s, xr_mul(a.r, c)), xr_fma(a.r, ns, xr_mul(a.i, c))};
}
// a (c + S i s) for constants c, s
template <int S> __device__ __forceinline__ X2C xrot(X2C a, float c, float s)
{
    const f32x2 C = x2_dup(c), P = x2_dup(s), N = x2_dup(-s);
    return S > 0 ? xmul(a, C, P, N) : xmulc(a, C, P, N);
}
// a times a table entry t = c + i s: a t (CONJ: a conj(t))
template <bool CONJ> __device__ __forceinline__ X2C xmul_tab(X2C a, float2 t)
{
    const f32x2 c = x2_dup(t.x), s = x2_dup(t.y);
    const f32x2 ns = xr_sub(0ull, s);
    return CONJ ? xmulc(a, c, s, ns) : xmul(a, c, s, ns);
}

// DFT4 of sign S; ROT2: the third input enters multiplied by S i (folded into the sums).
template <int S, bool ROT2 = false> __device__ __forceinline__ void xdft4(X2C &x0, X2C &x1, X2C &x2, X2C &x3)
{
    X2C t0, t1;
    if (!ROT2) {
        t0 = xadd(x0, x2);
        t1 = xsub(x0, x2);
    } else if (S > 0) {  // x2 i = (-x2.i, x2.r)
        t0 = X2C{xr_sub(x0.r, x2.i), xr_add(x0.i, x2.r)};
        t1 = X2C{xr_add(x0.r, x2.i), xr_sub(x0.i, x2.r)};
    } else {  // x2 (-i) = (x2.i, -x2.r)
        t0 = X2C{xr_add(x0.r, x2.i), xr_sub(x0.i, x2.r)};
        t1 = X2C{xr_sub(x0.r, x2.i), xr_add(x0.i, x2.r)};
    }
    const X2C t2 = xadd(x1, x3), d = xsub(x1, x3);
    x0 = xadd(t0, t2);
    x2 = xsub(t0, t2);
    // t3 = d (S i): x1 = t1 + t3, x3 = t1 - t3
    if (S > 0) {
        x1 = X2C{xr_sub(t1.r, d.i), xr_add(t1.i, d.r)};
        x3 = X2C{xr_add(t1.r, d.i), xr_sub(t1.i, d.r)};
    } else {
        x1 = X2C{xr_add(t1.r, d.i), xr_sub(t1.i, d.r)};
        x3 = X2C{xr_sub(t1.r, d.i), xr_add(t1.i, d.r)};
    }
}

template <int R, int S> struct XDft;

// 8 = 2 x 4: a_m = x_m + x_{m+4}, b_m = (x_m - x_{m+4}) W8^m, y_{2k} = DFT4(a), y_{2k+1} = DFT4(b)
template <int S> struct XDft<8, S> {
    __device__ __forceinline__ static void run(X2C *x)
    {
        const float r2 = Roots<float>::r2;
        X2C a0 = xadd(x[0], x[4]), a1 = xadd(x[1], x[5]), a2 = xadd(x[2], x[6]), a3 = xadd(x[3], x[7]);
        X2C b0 = xsub(x[0], x[4]);
        X2C b1 = xrot<S>(xsub(x[1], x[5]), r2, r2);
        X2C b2 = xsub(x[2], x[6]);  // enters DFT4(b) times S i
        X2C b3 = xrot<S>(xsub(x[3], x[7]), -r2, r2);
        xdft4<S>(a0, a1, a2, a3);
        xdft4<S, true>(b0, b1, b2, b3);
        x[0] = a0; x[2] = a1; x[4] = a2; x[6] = a3;
        x[1] = b0; x[3] = b1; x[5] = b2; x[7] = b3;
    }
};

// 16 = 4 x 4: u_{m,r} = DFT4_j(x_{m+4j})_r, u_{m,r} *= W16^{m r}, y_{4k+r} = DFT4_m(u_{m,r})_k
template <int S> struct XDft<16, S> {
    __device__ __forceinline__ static void run(X2C *x)
    {
        const float r2 = Roots<float>::r2, c8 = Roots<float>::c8, s8 = Roots<float>::s8;
#pragma unroll
        for (int m = 0; m < 4; m++) xdft4<S>(x[m], x[m + 4], x[m + 8], x[m + 12]);
        x[1 + 4 * 1] = xrot<S>(x[1 + 4 * 1], c8, s8);    // W^1
        x[1 + 4 * 2] = xrot<S>(x[1 + 4 * 2], r2, r2);    // W^2
        x[1 + 4 * 3] = xrot<S>(x[1 + 4 * 3], s8, c8);    // W^3
        x[2 + 4 * 1] = xrot<S>(x[2 + 4 * 1], r2, r2);    // W^2
        // x[2 + 4 * 2] times W^4 = S i: folded into its DFT4 below
        x[2 + 4 * 3] = xrot<S>(x[2 + 4 * 3], -r2, r2);   // W^6
        x[3 + 4 * 1] = xrot<S>(x[3 + 4 * 1], s8, c8);    // W^3
        x[3 + 4 * 2] = xrot<S>(x[3 + 4 * 2], -r2, r2);   // W^6
        x[3 + 4 * 3] = xrot<S>(x[3 + 4 * 3], -c8, -s8);  // W^9
        xdft4<S>(x[0], x[1], x[2], x[3]);
        xdft4<S>(x[4], x[5], x[6], x[7]);
        xdft4<S, true>(x[8], x[9], x[10], x[11]);
        xdft4<S>(x[12], x[13], x[14], x[15]);
        // x[4 r + k] = y_{4 k + r}: transpose the 4 x 4 block (register renaming)
        X2C t;
        t = x[1]; x[1] = x[4]; x[4] = t;
        t = x[2]; x[2] = x[8]; x[8] = t;
        t = x[3]; x[3] = x[12]; x[12] = t;
        t = x[6]; x[6] = x[9]; x[9] = t;
        t = x[7]; x[7] = x[13]; x[13] = t;
        t = x[11]; x[11] = x[14]; x[14] = t;
    }
};

template <int R, int S> __device__ __forceinline__ void xdft(X2C *x) { XDft<R, S>::run(x); }

__device__ __forceinline__ X2C lds_x2c(const float2 *p)
{
    const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p);
    return X2C{v.x, v.y};
}
__device__ __forceinline__ void sts_x2c(float2 *p, X2C v) { *reinterpret_cast<ulonglong2 *>(p) = make_ulonglong2(v.r, v.i); }
// Interleaved pixel pair {re_l, im_l, re_l+1, im_l+1} <-> split pair
__device__ __forceinline__ X2C split_of(float4 q)
{
    return X2C{f2pack(float2{q.x, q.z}), f2pack(float2{q.y, q.w})};
}
__device__ __forceinline__ float4 interleaved_of(X2C v)
{
    const float2 re = f2unpack(v.r), im = f2unpack(v.i);
    return make_float4(re.x, im.x, re.y, im.y);
}

template <int NT, int RA> struct LineGeom {
    static constexpr int RB = NT / RA;
    static constexpr int Q = RB;  // butterflies per line of the RA-point stage
    static constexpr int PP = kLineP / 2;  // pixel pairs per row
    static constexpr int ROWS = NT + NT / RB;
    static constexpr int REGION = ROWS * kLineP;  // float2 elements per field region
    __device__ __forceinline__ static constexpr int row(int t) { return t + t / RB; }
    static constexpr size_t smem_bytes() { return 3 * (size_t)REGION * sizeof(float2); }
};

template <int NT, int RA> struct LineItems {
    static constexpr int A = LineGeom<NT, RA>::PP * LineGeom<NT, RA>::Q;  // RA-point butterflies per field
    static constexpr int B = LineGeom<NT, RA>::PP * RA;                   // RB-point butterflies per field
};

// Item w of field f in the forward RA-point stage (stride Q): butterfly, then the
// twiddles W_NT^{j k}.
template <int NT, int RA>
__device__ __forceinline__ void line_stage_a(const TPassArgs<float2> &a, float2 *sm, int f, int w)
{
    using G = LineGeom<NT, RA>;
    constexpr int Q = G::Q, PP = G::PP;
    const int pp = w % PP, j = w / PP;
    float2 *sp = sm + f * G::REGION + 2 * pp;
    X2C x[RA];
#pragma unroll
    for (int m = 0; m < RA; m++) x[m] = lds_x2c(sp + G::row(j + Q * m) * kLineP);
    xdft<RA, +1>(x);
#pragma unroll
    for (int k = 1; k < RA; k++) x[k] = xmul_tab<true>(x[k], __ldg(a.tw + (k - 1) * Q + j));
#pragma unroll
    for (int k = 0; k < RA; k++) sts_x2c(sp + G::row(j + Q * k) * kLineP, x[k]);
}

// Item w of field f in the RB-point stage: butterfly, phase table, inverse butterfly.
template <int NT, int RA>
__device__ __forceinline__ void line_stage_b(const TPassArgs<float2> &a, float2 *sm, int f, int w)
{
    using G = LineGeom<NT, RA>;
    constexpr int RB = G::RB, PP = G::PP;
    const int pp = w % PP, g = w / PP;
    float2 *sp = sm + f * G::REGION + G::row(RB * g) * kLineP + 2 * pp;
    const float2 *tb = a.tab[f] + RB * g;
    X2C x[RB];
#pragma unroll
    for (int m = 0; m < RB; m++) x[m] = lds_x2c(sp + m * kLineP);
    xdft<RB, +1>(x);
#pragma unroll
    for (int k = 0; k < RB; k++) x[k] = xmul_tab<false>(x[k], __ldg(tb + k));
    xdft<RB, -1>(x);
#pragma unroll
    for (int k = 0; k < RB; k++) sts_x2c(sp + k * kLineP, x[k]);
}

// Item w of field f in the inverse RA-point stage (twiddles before the butterfly),
// written to global memory.
template <int NT, int RA>
__device__ __forceinline__ void line_stage_c(const TPassArgs<float2> &a, const float2 *sm, int f, int w,
                                             unsigned base, unsigned gs)
{
    using G = LineGeom<NT, RA>;
    constexpr int Q = G::Q, PP = G::PP;
    const int pp = w % PP, j = w / PP;
    const float2 *sp = sm + f * G::REGION + 2 * pp;
    X2C x[RA];
#pragma unroll
    for (int m = 0; m < RA; m++) x[m] = lds_x2c(sp + G::row(j + Q * m) * kLineP);
#pragma unroll
    for (int m = 1; m < RA; m++) x[m] = xmul_tab<false>(x[m], __ldg(a.tw + (m - 1) * Q + j));
    xdft<RA, -1>(x);
    float2 *d = a.f[f] + base + (unsigned)j * gs + 2 * pp;
#pragma unroll
    for (int k = 0; k < RA; k++) *reinterpret_cast<float4 *>(d + (size_t)(Q * k) * gs) = interleaved_of(x[k]);
}

// One tile: P = 8 consecutive pixels of one row, all NT samples, the fields in the load
// mask, staged with cp.async; coupled-wave half steps (and the EOM) as a sweep over the
// tile; then per transformed field the RA-point stage, the fused RB-point stage with the
// phase table, and the inverse RA-point stage written to global memory.
template <int NT, int RA, int THREADS, int BAR = 0>
__device__ __forceinline__ void tpass_line_tile(const TPassArgs<float2> &a, unsigned tile, float2 *sm)
{
    using G = LineGeom<NT, RA>;
    constexpr int PP = G::PP;
    const unsigned base = tile_base(a.g, tile);
    const unsigned gs = a.g.gs_j;  // nx ny: one time sample
    const unsigned tmask = a.tmask;
    const unsigned lmask = tpass_load_mask(a);

    // stage the tile: 16-byte copies of pixel pairs, interleaved as in global memory
    {
        const float2 *src[3] = {a.psrc, a.f[1], a.f[2]};
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (!(lmask & (1u << f))) continue;
            const float2 *gsrc = src[f] + base;
            float2 *dst = sm + f * G::REGION;
            for (int e = threadIdx.x; e < NT * PP; e += THREADS) {
                const int t = e / PP, pp = e % PP;
                cp_async<16>(dst + G::row(t) * kLineP + 2 * pp, gsrc + (size_t)t * gs + 2 * pp);
            }
        }
        cp_async_wait_all();
        tile_sync<BAR>();
    }

    // sweep: half steps and EOM per voxel pair; transformed fields go back to shared
    // memory as split pairs, the others (loaded, not transformed) to global memory
    for (int e = threadIdx.x; e < NT * PP; e += THREADS) {
        const int t = e / PP, pp = e % PP;
        const int off = G::row(t) * kLineP + 2 * pp;
        f32x2 v[3][2];
#pragma unroll
        for (int f = 0; f < 3; f++) {
            float4 q4 = make_float4(0.f, 0.f, 0.f, 0.f);
            if (lmask & (1u << f)) q4 = *reinterpret_cast<const float4 *>(sm + f * G::REGION + off);
            const X2C x = split_of(q4);
            v[f][0] = x.r;
            v[f][1] = x.i;
        }
        if (!a.use_phase) {
            for (int h = 0; h < a.n_rk4; h++) rk4_half_fast_x2(a, v[0], v[1], v[2]);
        } else if (a.n_rk4 > 0) {
            // corrected physics with a phase mismatch: per voxel
            float2 u[2][3];
#pragma unroll
            for (int f = 0; f < 3; f++) {
                const float2 re = f2unpack(v[f][0]), im = f2unpack(v[f][1]);
                u[0][f] = float2{re.x, im.x};
                u[1][f] = float2{re.y, im.y};
            }
            for (int h = 0; h < a.n_rk4; h++) {
                rk4_half(a, h, u[0][0], u[0][1], u[0][2]);
                rk4_half(a, h, u[1][0], u[1][1], u[1][2]);
            }
#pragma unroll
            for (int f = 0; f < 3; f++) {
                v[f][0] = f2pack(float2{u[0][f].x, u[1][f].x});
                v[f][1] = f2pack(float2{u[0][f].y, u[1][f].y});
            }
        }
        if (a.eom) {
            const float2 ev = __ldg(a.eom + t);
            const f32x2 er = x2_dup(ev.x), ei = x2_dup(ev.y), nei = x2_dup(-ev.y);
#pragma unroll
            for (int f = 1; f < 3; f++) {
                const X2C y = xmul(X2C{v[f][0], v[f][1]}, er, ei, nei);
                v[f][0] = y.r;
                v[f][1] = y.i;
            }
        }
        const unsigned gb = base + (unsigned)t * gs + 2 * pp;
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (tmask & (1u << f))
                sts_x2c(sm + f * G::REGION + off, X2C{v[f][0], v[f][1]});
            else if (lmask & (1u << f))
                *reinterpret_cast<float4 *>(a.f[f] + gb) = interleaved_of(X2C{v[f][0], v[f][1]});
        }
    }
    if (!tmask) {
        tile_sync<BAR>();
        return;
    }
    tile_sync<BAR>();
    const int nf = __popc(tmask);
    if constexpr (THREADS == 32 * 3) {
        // one warp per transformed field: its three stages synchronise the warp only
        const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (wid < nf) {
            const int f = field_id(tmask, wid);
#pragma unroll
            for (int w = lane; w < LineItems<NT, RA>::A; w += 32) line_stage_a<NT, RA>(a, sm, f, w);
            __syncwarp();
#pragma unroll
            for (int w = lane; w < LineItems<NT, RA>::B; w += 32) line_stage_b<NT, RA>(a, sm, f, w);
            __syncwarp();
#pragma unroll
            for (int w = lane; w < LineItems<NT, RA>::A; w += 32) line_stage_c<NT, RA>(a, sm, f, w, base, gs);
        }
    } else {
        constexpr int IA = LineItems<NT, RA>::A, IB = LineItems<NT, RA>::B;
        for (int u = threadIdx.x; u < nf * IA; u += THREADS) line_stage_a<NT, RA>(a, sm, field_id(tmask, u / IA), u % IA);
        tile_sync<BAR>();
        for (int u = threadIdx.x; u < nf * IB; u += THREADS) line_stage_b<NT, RA>(a, sm, field_id(tmask, u / IB), u % IB);
        tile_sync<BAR>();
        for (int u = threadIdx.x; u < nf * IA; u += THREADS)
            line_stage_c<NT, RA>(a, sm, field_id(tmask, u / IA), u % IA, base, gs);
    }
    tile_sync<BAR>();
}

}  // namespace opo
