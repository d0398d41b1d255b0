// Register-resident radix butterflies for the in-shared-memory line FFTs of the split-
// step passes.  Each dft<R, S>(x) overwrites x[0..R) with
//   y[k] = sum_m x[m] exp(S 2 pi i m k / R),  S = +1 or -1, unnormalised,
// in natural order.  Written from the DFT definition with the usual radix-2/4
// decimation identities; the only constants are the R-th roots of unity.
#pragma once

#include <cuda_runtime.h>

namespace opo {

template <typename T> struct Cpx;
template <> struct Cpx<float> { using type = float2; };
template <> struct Cpx<double> { using type = double2; };

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return C{a.x + b.x, a.y + b.y}; }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return C{a.x - b.x, a.y - b.y}; }
// float2: both components in one of Blackwell's packed two-lane FP32 instructions
// (add / sub .f32x2 on a 64-bit register pair), half the issue slots of two scalar ones.
__host__ __device__ __forceinline__ unsigned long long f2pack(float2 a)
{
#if defined(__CUDA_ARCH__)
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
#else
    return 0;
#endif
}
__host__ __device__ __forceinline__ float2 f2unpack(unsigned long long r)
{
    float2 a{0.f, 0.f};
#if defined(__CUDA_ARCH__)
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
#endif
    return a;
}
template <> __host__ __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("add.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(d);
#else
    return float2{a.x + b.x, a.y + b.y};
#endif
}
template <> __host__ __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b)
{
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("sub.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2pack(a)), "l"(f2pack(b)));
    return f2unpack(d);
#else
    return float2{a.x - b.x, a.y - b.y};
#endif
}
// y + s x for real s
template <typename C, typename T> __host__ __device__ __forceinline__ C caxpy(T s, C x, C y)
{
    return C{y.x + s * x.x, y.y + s * x.y};
}
template <> __host__ __device__ __forceinline__ float2 caxpy<float2, float>(float s, float2 x, float2 y)
{
#if defined(__CUDA_ARCH__)
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2pack(float2{s, s})), "l"(f2pack(x)), "l"(f2pack(y)));
    return f2unpack(d);
#else
    return float2{y.x + s * x.x, y.y + s * x.y};
#endif
}
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b)
{
    return C{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b)
{
    return C{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename C, typename T> __host__ __device__ __forceinline__ C cscale(C a, T s) { return C{a.x * s, a.y * s}; }
// a * (S i)
template <int S, typename C> __host__ __device__ __forceinline__ C cmul_si(C a)
{
    return S > 0 ? C{-a.y, a.x} : C{a.y, -a.x};
}
// a * (c + S i s) for real c, s
template <int S, typename C, typename T> __host__ __device__ __forceinline__ C cmul_cs(C a, T c, T s)
{
    return S > 0 ? C{a.x * c - a.y * s, a.x * s + a.y * c} : C{a.x * c + a.y * s, a.y * c - a.x * s};
}

// Root-of-unity constants (values of cos and sin at multiples of pi/8 and pi/3).
template <typename T> struct Roots {
    static constexpr T r2 = T(0.70710678118654752440);  // cos(pi/4)
    static constexpr T c8 = T(0.92387953251128675613);  // cos(pi/8)
    static constexpr T s8 = T(0.38268343236508977173);  // sin(pi/8)
    static constexpr T s3 = T(0.86602540378443864676);  // sin(pi/3)
};

template <int S, typename C> __host__ __device__ __forceinline__ void dft2(C &a, C &b)
{
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int S, typename C> __host__ __device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3)
{
    C t0 = cadd(x0, x2), t1 = csub(x0, x2);
    C t2 = cadd(x1, x3), t3 = cmul_si<S>(csub(x1, x3));
    x0 = cadd(t0, t2);
    x2 = csub(t0, t2);
    x1 = cadd(t1, t3);
    x3 = csub(t1, t3);
}

template <int R, int S, typename C> struct Dft;

template <int S, typename C> struct Dft<2, S, C> {
    __host__ __device__ __forceinline__ static void run(C *x) { dft2<S>(x[0], x[1]); }
};

template <int S, typename C> struct Dft<3, S, C> {
    __host__ __device__ __forceinline__ static void run(C *x)
    {
        using T = decltype(x[0].x);
        C t1 = cadd(x[1], x[2]);
        C t2 = cmul_si<S>(cscale(csub(x[1], x[2]), Roots<T>::s3));
        C m = csub(x[0], cscale(t1, T(0.5)));
        x[0] = cadd(x[0], t1);
        x[1] = cadd(m, t2);
        x[2] = csub(m, t2);
    }
};

template <int S, typename C> struct Dft<4, S, C> {
    __host__ __device__ __forceinline__ static void run(C *x) { dft4<S>(x[0], x[1], x[2], x[3]); }
};

// 8 = 2 x 4: a_m = x_m + x_{m+4}, b_m = (x_m - x_{m+4}) W8^m, y_{2k} = DFT4(a), y_{2k+1} = DFT4(b)
template <int S, typename C> struct Dft<8, S, C> {
    __host__ __device__ __forceinline__ static void run(C *x)
    {
        using T = decltype(x[0].x);
        const T r2 = Roots<T>::r2;
        C a0 = cadd(x[0], x[4]), a1 = cadd(x[1], x[5]), a2 = cadd(x[2], x[6]), a3 = cadd(x[3], x[7]);
        C b0 = csub(x[0], x[4]);
        C b1 = cmul_cs<S>(csub(x[1], x[5]), r2, r2);
        C b2 = cmul_si<S>(csub(x[2], x[6]));
        C b3 = cmul_cs<S>(csub(x[3], x[7]), -r2, r2);
        dft4<S>(a0, a1, a2, a3);
        dft4<S>(b0, b1, b2, b3);
        x[0] = a0; x[2] = a1; x[4] = a2; x[6] = a3;
        x[1] = b0; x[3] = b1; x[5] = b2; x[7] = b3;
    }
};

// 16 = 4 x 4: u_{m,r} = DFT4_j(x_{m+4j})_r, u_{m,r} *= W16^{m r}, y_{4k+r} = DFT4_m(u_{m,r})_k
template <int S, typename C> struct Dft<16, S, C> {
    __host__ __device__ __forceinline__ static void run(C *x)
    {
        using T = decltype(x[0].x);
        const T r2 = Roots<T>::r2, c8 = Roots<T>::c8, s8 = Roots<T>::s8;
#pragma unroll
        for (int m = 0; m < 4; m++) dft4<S>(x[m], x[m + 4], x[m + 8], x[m + 12]);
        // after this x[m + 4 r] = u_{m,r}
        x[1 + 4 * 1] = cmul_cs<S>(x[1 + 4 * 1], c8, s8);    // W^1
        x[1 + 4 * 2] = cmul_cs<S>(x[1 + 4 * 2], r2, r2);    // W^2
        x[1 + 4 * 3] = cmul_cs<S>(x[1 + 4 * 3], s8, c8);    // W^3
        x[2 + 4 * 1] = cmul_cs<S>(x[2 + 4 * 1], r2, r2);    // W^2
        x[2 + 4 * 2] = cmul_si<S>(x[2 + 4 * 2]);             // W^4
        x[2 + 4 * 3] = cmul_cs<S>(x[2 + 4 * 3], -r2, r2);   // W^6
        x[3 + 4 * 1] = cmul_cs<S>(x[3 + 4 * 1], s8, c8);    // W^3
        x[3 + 4 * 2] = cmul_cs<S>(x[3 + 4 * 2], -r2, r2);   // W^6
        x[3 + 4 * 3] = cmul_cs<S>(x[3 + 4 * 3], -c8, -s8);  // W^9
#pragma unroll
        for (int r = 0; r < 4; r++) dft4<S>(x[4 * r], x[4 * r + 1], x[4 * r + 2], x[4 * r + 3]);
        // now x[4 r + k] = y_{4 k + r}: transpose the 4 x 4 block in registers
        C t;
        t = x[1]; x[1] = x[4]; x[4] = t;
        t = x[2]; x[2] = x[8]; x[8] = t;
        t = x[3]; x[3] = x[12]; x[12] = t;
        t = x[6]; x[6] = x[9]; x[9] = t;
        t = x[7]; x[7] = x[13]; x[13] = t;
        t = x[11]; x[11] = x[14]; x[14] = t;
    }
};

template <int R, int S, typename C> __host__ __device__ __forceinline__ void dft(C *x) { Dft<R, S, C>::run(x); }

}  // namespace opo
