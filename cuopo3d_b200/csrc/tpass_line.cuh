// Line-specialised t-pass: the tile body of tpass_tile / tpass_tile_split for a time
// axis whose length and radix plan are compile-time constants (NT = RA x RB with RA, RB
// in {8, 16}: 64, 128, 256), in FP32 and FP64.
//
// It computes what the generic t-pass computes (reference Solver3D.cuh:872-943 RK4 half
// steps, then Solver3D.cuh:572-639 dispersion: transform, phase, inverse transform) on
// tiles of 16-byte units: four units per time sample, one time sample per shared-memory
// row.  A unit is one FP64 pixel, or in FP32 a split pair: the same time sample of
// pixels l and l + 1, real parts in one packed f32x2 register pair and imaginary parts
// in another, in registers and in shared memory (re_l, re_l+1, im_l, im_l+1).  Every FP32
// butterfly, twiddle and phase product then serves two lines with one packed instruction
// per component (a complex product: 4 packed instructions for two values; multiplying by
// +-i only renames registers), each twiddle and phase factor is loaded once for both
// lines, and all index arithmetic is compile-time.  A tile is 8 pixels (FP32) or 4
// (FP64) of one row.  The transforms are the generic two-stage plan [RA, RB] (decimation
// in frequency forward, in time inverse, phase tables in the plan's digit-reversed
// order), so the twiddles and phase tables are the host's tables of that plan.
//
// Shared memory per field: NT + NT / RB rows of four units; time sample t sits in row
// t + t / RB (a padding row after every RB rows), so the RB-point stage's eight
// butterflies of a warp fall on alternating halves of the banks, and the other stages
// read whole 512-byte runs.  The first stage's twiddles are staged with the tile, after
// the three field regions (shared-memory latency instead of L1 for the 30 twiddle loads
// of a first- and last-stage item; the phase tables stay in global memory).
//
// The single-instance kernel runs one tile per CTA, four CTAs of 128 threads per SM; the
// batched kernel runs the same body over the tiles of every instance.
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

__device__ __forceinline__ X2C split_of(float4 q)
{
    return X2C{f2pack(float2{q.x, q.z}), f2pack(float2{q.y, q.w})};
}
__device__ __forceinline__ float4 interleaved_of(X2C v)
{
    const float2 re = f2unpack(v.r), im = f2unpack(v.i);
    return make_float4(re.x, im.x, re.y, im.y);
}

// The 16-byte unit of each precision: its register form, loads and stores of the raw
// layout (the global one, C values interleaved: staged tiles and the fields), the
// butterflies, table products and the coupled-wave half steps.
template <typename C> struct LineUnit;

template <> struct LineUnit<float2> {
    using U = X2C;
    static constexpr int PX = 2;  // pixels per unit
    __device__ __forceinline__ static U lds(const void *p)
    {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(p);
        return X2C{v.x, v.y};
    }
    __device__ __forceinline__ static void sts(void *p, U v) { *reinterpret_cast<ulonglong2 *>(p) = make_ulonglong2(v.r, v.i); }
    __device__ __forceinline__ static U load_raw(const void *p) { return split_of(*reinterpret_cast<const float4 *>(p)); }
    __device__ __forceinline__ static void store_raw(void *p, U v) { *reinterpret_cast<float4 *>(p) = interleaved_of(v); }
    template <int R, int S> __device__ __forceinline__ static void dft(U *x) { xdft<R, S>(x); }
    // x t (CONJ: x conj(t)) for a table entry t
    template <bool CONJ> __device__ __forceinline__ static U tmul(U x, float2 t) { return xmul_tab<CONJ>(x, t); }
    __device__ __forceinline__ static U zero() { return X2C{0ull, 0ull}; }
    // n half steps of every voxel of the units p, s, i
    __device__ __forceinline__ static void rk4(const TPassArgs<float2> &a, U &p, U &s, U &i)
    {
        if (!a.use_phase) {
            f32x2 v[3][2] = {{p.r, p.i}, {s.r, s.i}, {i.r, i.i}};
            for (int h = 0; h < a.n_rk4; h++) rk4_half_fast_x2(a, v[0], v[1], v[2]);
            p = X2C{v[0][0], v[0][1]};
            s = X2C{v[1][0], v[1][1]};
            i = X2C{v[2][0], v[2][1]};
            return;
        }
        // corrected physics with a phase mismatch: per voxel
        U *u[3] = {&p, &s, &i};
        float2 w[2][3];
#pragma unroll
        for (int f = 0; f < 3; f++) {
            const float2 re = f2unpack(u[f]->r), im = f2unpack(u[f]->i);
            w[0][f] = float2{re.x, im.x};
            w[1][f] = float2{re.y, im.y};
        }
        for (int h = 0; h < a.n_rk4; h++) {
            rk4_half(a, h, w[0][0], w[0][1], w[0][2]);
            rk4_half(a, h, w[1][0], w[1][1], w[1][2]);
        }
#pragma unroll
        for (int f = 0; f < 3; f++) *u[f] = X2C{f2pack(float2{w[0][f].x, w[1][f].x}), f2pack(float2{w[0][f].y, w[1][f].y})};
    }
};

template <> struct LineUnit<double2> {
    using U = double2;
    static constexpr int PX = 1;
    __device__ __forceinline__ static U lds(const void *p) { return *reinterpret_cast<const double2 *>(p); }
    __device__ __forceinline__ static void sts(void *p, U v) { *reinterpret_cast<double2 *>(p) = v; }
    __device__ __forceinline__ static U load_raw(const void *p) { return *reinterpret_cast<const double2 *>(p); }
    __device__ __forceinline__ static void store_raw(void *p, U v) { *reinterpret_cast<double2 *>(p) = v; }
    template <int R, int S> __device__ __forceinline__ static void dft(U *x) { opo::dft<R, S>(x); }
    template <bool CONJ> __device__ __forceinline__ static U tmul(U x, double2 t) { return CONJ ? cmulc(x, t) : cmul(x, t); }
    __device__ __forceinline__ static U zero() { return double2{0.0, 0.0}; }
    __device__ __forceinline__ static void rk4(const TPassArgs<double2> &a, U &p, U &s, U &i)
    {
        for (int h = 0; h < a.n_rk4; h++) rk4_half(a, h, p, s, i);
    }
};

template <typename C, int NT, int RA> struct LineGeom {
    static constexpr int RB = NT / RA;
    static constexpr int Q = RB;  // butterflies per line of the RA-point stage
    static constexpr int PP = 4;  // units per row (time sample)
    static constexpr int P = PP * LineUnit<C>::PX;  // pixels per tile
    static constexpr int ROWS = NT + NT / RB;
    static constexpr int REGION = ROWS * PP * 16;  // bytes per field region
    static constexpr int A = PP * Q;   // RA-point butterflies per field
    static constexpr int B = PP * RA;  // RB-point butterflies per field
    __device__ __forceinline__ static constexpr int row(int t) { return t + t / RB; }
    // byte offset of (field f, time sample t, unit u) in a tile buffer
    __device__ __forceinline__ static constexpr int at(int f, int t, int u) { return f * REGION + (row(t) * PP + u) * 16; }
    static constexpr int NTW = (RA - 1) * Q;  // first-stage twiddles, staged after the tile
    static constexpr int TILE_BYTES = 3 * REGION;
    static constexpr size_t tile_bytes() { return (size_t)TILE_BYTES + (size_t)NTW * sizeof(C); }
};

// Issue the cp.async copies of tile `tile` (the fields in lmask) into buffer buf.
template <typename C, int NT, int RA, int THREADS>
__device__ __forceinline__ void line_stage_in(const TPassArgs<C> &a, unsigned tile, unsigned lmask, unsigned char *buf)
{
    using G = LineGeom<C, NT, RA>;
    const unsigned base = tile_base(a.g, tile), gs = a.g.gs_j;
    const C *src[3] = {a.psrc, a.f[1], a.f[2]};
#pragma unroll
    for (int f = 0; f < 3; f++) {
        if (!(lmask & (1u << f))) continue;
        const C *gsrc = src[f] + base;
        for (unsigned e = threadIdx.x; e < NT * G::PP; e += THREADS) {
            const int t = (int)(e / G::PP), u = (int)(e % G::PP);
            cp_async<16>(buf + G::at(f, t, u), gsrc + (size_t)t * gs + u * LineUnit<C>::PX);
        }
    }
}

// Sweep over the staged tile: half steps and EOM per unit, two units per thread at a time
// (items e and e + THREADS: two independent chains to interleave); transformed fields go
// back to shared memory as units, the others (loaded, not transformed) to global memory.
template <typename C, int NT, int RA, int THREADS>
__device__ __forceinline__ void line_sweep(const TPassArgs<C> &a, unsigned base, unsigned lmask, unsigned tmask,
                                           unsigned char *buf)
{
    using G = LineGeom<C, NT, RA>;
    using L = LineUnit<C>;
    using U = typename L::U;
    const unsigned gs = a.g.gs_j;
    auto load = [&](unsigned e, U (&v)[3]) {
        const int t = (int)(e / G::PP), u = (int)(e % G::PP);
#pragma unroll
        for (int f = 0; f < 3; f++) v[f] = (lmask & (1u << f)) ? L::load_raw(buf + G::at(f, t, u)) : L::zero();
    };
    auto finish = [&](unsigned e, U (&v)[3]) {
        const int t = (int)(e / G::PP), u = (int)(e % G::PP);
        if (a.eom) {
            const C ev = __ldg(a.eom + t);
            v[1] = L::template tmul<false>(v[1], ev);
            v[2] = L::template tmul<false>(v[2], ev);
        }
#pragma unroll
        for (int f = 0; f < 3; f++) {
            if (tmask & (1u << f))
                L::sts(buf + G::at(f, t, u), v[f]);
            else if (lmask & (1u << f))
                L::store_raw(a.f[f] + base + (unsigned)t * gs + u * L::PX, v[f]);
        }
    };
    constexpr unsigned NI = NT * G::PP;
    for (unsigned e = threadIdx.x; e < NI; e += 2 * THREADS) {
        const bool two = e + THREADS < NI;
        U v0[3], v1[3];
        load(e, v0);
        if (two) load(e + THREADS, v1);
        L::rk4(a, v0[0], v0[1], v0[2]);
        if (two) L::rk4(a, v1[0], v1[1], v1[2]);
        finish(e, v0);
        if (two) finish(e + THREADS, v1);
    }
}

// Item w of field f in the forward RA-point stage (stride Q): butterfly, then the
// twiddles W_NT^{j k}.
template <typename C, int NT, int RA>
__device__ __forceinline__ void line_stage_a(const TPassArgs<C> &a, unsigned char *buf, int f, unsigned w)
{
    using G = LineGeom<C, NT, RA>;
    using L = LineUnit<C>;
    constexpr int Q = G::Q;
    const int u = (int)(w % G::PP), j = (int)(w / G::PP);
    typename L::U x[RA];
#pragma unroll
    for (int m = 0; m < RA; m++) x[m] = L::lds(buf + G::at(f, j + Q * m, u));
    L::template dft<RA, +1>(x);
    const C *tws = reinterpret_cast<const C *>(buf + G::TILE_BYTES);
#pragma unroll
    for (int k = 1; k < RA; k++) x[k] = L::template tmul<true>(x[k], tws[(k - 1) * Q + j]);
#pragma unroll
    for (int k = 0; k < RA; k++) L::sts(buf + G::at(f, j + Q * k, u), x[k]);
}

// Item w of field f in the RB-point stage: butterfly, phase table, inverse butterfly.
template <typename C, int NT, int RA>
__device__ __forceinline__ void line_stage_b(const TPassArgs<C> &a, unsigned char *buf, int f, unsigned w)
{
    using G = LineGeom<C, NT, RA>;
    using L = LineUnit<C>;
    constexpr int RB = G::RB;
    const int u = (int)(w % G::PP), g = (int)(w / G::PP);
    unsigned char *sp = buf + G::at(f, RB * g, u);
    const C *tb = a.tab[f] + RB * g;
    typename L::U x[RB];
#pragma unroll
    for (int m = 0; m < RB; m++) x[m] = L::lds(sp + m * G::PP * 16);
    L::template dft<RB, +1>(x);
    if constexpr (sizeof(C) == 8) {
        // two FP32 table entries per 16-byte load (tb is 16-byte aligned: RB g even)
#pragma unroll
        for (int k = 0; k < RB; k += 2) {
            const float4 t2 = __ldg(reinterpret_cast<const float4 *>(tb + k));
            x[k] = L::template tmul<false>(x[k], C{t2.x, t2.y});
            x[k + 1] = L::template tmul<false>(x[k + 1], C{t2.z, t2.w});
        }
    } else {
#pragma unroll
        for (int k = 0; k < RB; k++) x[k] = L::template tmul<false>(x[k], __ldg(tb + k));
    }
    L::template dft<RB, -1>(x);
#pragma unroll
    for (int k = 0; k < RB; k++) L::sts(sp + k * G::PP * 16, x[k]);
}

// Item w of field f in the inverse RA-point stage (twiddles before the butterfly),
// written to global memory.
template <typename C, int NT, int RA>
__device__ __forceinline__ void line_stage_c(const TPassArgs<C> &a, const unsigned char *buf, int f, unsigned w,
                                             unsigned base, unsigned gs)
{
    using G = LineGeom<C, NT, RA>;
    using L = LineUnit<C>;
    constexpr int Q = G::Q;
    const int u = (int)(w % G::PP), j = (int)(w / G::PP);
    typename L::U x[RA];
#pragma unroll
    for (int m = 0; m < RA; m++) x[m] = L::lds(buf + G::at(f, j + Q * m, u));
    const C *tws = reinterpret_cast<const C *>(buf + G::TILE_BYTES);
#pragma unroll
    for (int m = 1; m < RA; m++) x[m] = L::template tmul<false>(x[m], tws[(m - 1) * Q + j]);
    L::template dft<RA, -1>(x);
    C *d = a.f[f] + base + (unsigned)j * gs + u * L::PX;
#pragma unroll
    for (int k = 0; k < RA; k++) L::store_raw(d + (size_t)(Q * k) * gs, x[k]);
}

// The three transform stages of every field in tmask as jobs (stage, field) in
// stage-major order, two jobs per phase (half the CTA each; one job when one field is
// transformed) and a CTA barrier between phases.  A job's stage of a field always ran
// in an earlier phase (nf >= 2 jobs apart), and three fields take five phases of whole
// warps instead of three stages that leave half the warps idle for their second half.
template <typename C, int NT, int RA, int THREADS, int BAR, int PER>
__device__ __forceinline__ void line_jobs(const TPassArgs<C> &a, unsigned base, unsigned tmask, unsigned nf,
                                          unsigned char *buf)
{
    using G = LineGeom<C, NT, RA>;
    constexpr unsigned GROUP = THREADS / PER;
    const unsigned gs = a.g.gs_j, njobs = 3 * nf;
    const unsigned slot = threadIdx.x / GROUP, w0 = threadIdx.x % GROUP;
    for (unsigned j0 = 0; j0 < njobs; j0 += PER) {
        const unsigned j = j0 + slot;
        if (j < njobs) {
            // stage j / nf and field j % nf for nf = 1, 2, 3 (j < 9: j / 3 = (11 j) >> 5)
            const unsigned stage = nf == 1 ? j : (nf == 2 ? j >> 1 : (11 * j) >> 5);
            const int f = field_id(tmask, (int)(j - stage * nf));
            if (stage == 0) {
                for (unsigned w = w0; w < G::A; w += GROUP) line_stage_a<C, NT, RA>(a, buf, f, w);
            } else if (stage == 1) {
                for (unsigned w = w0; w < G::B; w += GROUP) line_stage_b<C, NT, RA>(a, buf, f, w);
            } else {
                for (unsigned w = w0; w < G::A; w += GROUP) line_stage_c<C, NT, RA>(a, buf, f, w, base, gs);
            }
        }
        tile_sync<BAR>();
    }
}

template <typename C, int NT, int RA, int THREADS, int BAR>
__device__ __forceinline__ void line_transforms(const TPassArgs<C> &a, unsigned base, unsigned tmask, unsigned char *buf)
{
    const unsigned nf = __popc(tmask);
    if (nf >= 2)
        line_jobs<C, NT, RA, THREADS, BAR, 2>(a, base, tmask, nf, buf);
    else
        line_jobs<C, NT, RA, THREADS, BAR, 1>(a, base, tmask, nf, buf);
}

// One tile: the fields in the load mask staged with cp.async, the sweep, then per
// transformed field the RA-point stage, the fused RB-point stage with the phase table,
// and the inverse RA-point stage written to global memory.  Ends with the CTA
// synchronised.
template <typename C, int NT, int RA, int THREADS, int BAR = 0>
__device__ __forceinline__ void tpass_line_tile(const TPassArgs<C> &a, unsigned tile, unsigned char *buf)
{
    const unsigned base = tile_base(a.g, tile);
    const unsigned tmask = a.tmask, lmask = tpass_load_mask(a);
    line_stage_in<C, NT, RA, THREADS>(a, tile, lmask, buf);
    {  // the first stage's twiddles
        using G = LineGeom<C, NT, RA>;
        C *tws = reinterpret_cast<C *>(buf + G::TILE_BYTES);
        for (int e = threadIdx.x; e < G::NTW; e += THREADS) cp_async<sizeof(C)>(tws + e, a.tw + e);
    }
    cp_async_wait_all();
    tile_sync<BAR>();
    line_sweep<C, NT, RA, THREADS>(a, base, lmask, tmask, buf);
    tile_sync<BAR>();
    if (tmask) line_transforms<C, NT, RA, THREADS, BAR>(a, base, tmask, buf);
}

}  // namespace opo
