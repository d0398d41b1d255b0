// Gain compensation of the FP32 transform pairs (host code, shared by the solver's
// table builder and the host-side check in tests/native/gain_check.cu).
//
// The FP32 kernels' roots of unity -- the butterflies' constants (fft_radix.cuh) and the
// stage twiddles, computed in FP64 and rounded -- have |W|^2 - 1 of a few 1e-8, mostly
// negative, so forward transform -> phase table -> inverse transform is not exactly
// norm-preserving: it drains ~2e-8 of the energy per pass, coherently, every split step
// (about 5e-6 of the energy per 100-step round trip and pass kind).  Every input-output
// pair of a Cooley-Tukey network is joined by one chain of butterflies, so the squared
// row norms r_p of the forward operator and the squared column norms c_p of the inverse
// follow from running the network on squared magnitudes: r = |F|^2 1, c = (|F_inv|^2)^T 1.
// A pair with exact constants has r_p = c_p = n; a phase table scaled by n / sqrt(r_p c_p)
// at spectrum position p gives the pair the energy gain of the table itself for white
// inputs, which removes the coherent drain.  What remains is the arithmetic's own
// rounding.
#pragma once

#include "fft_radix.cuh"
#include "opo_internal.h"

#include <cmath>
#include <complex>
#include <vector>

namespace opo {

// |B_km|^2 of the radix-R butterfly as the FP32 kernels compute it: dft<R> run on float2
// unit vectors, whose outputs are exactly the FP32 constants (sums of them, for radix 3).
template <int R> inline void butterfly_sq(std::vector<double> &b2)
{
    b2.assign((size_t)R * R, 0.0);
    for (int m = 0; m < R; m++) {
        float2 x[R];
        for (int k = 0; k < R; k++) x[k] = make_float2(k == m ? 1.f : 0.f, 0.f);
        dft<R, +1>(x);
        for (int k = 0; k < R; k++) b2[(size_t)k * R + m] = (double)x[k].x * x[k].x + (double)x[k].y * x[k].y;
    }
}

// Per position of the digit-reversed spectrum: n / sqrt(r_p c_p) for plan pl, whose
// FP64 stage twiddles tw (AxisPlan layout) the kernels get rounded to FP32.
inline std::vector<double> fp32_pair_compensation(const AxisPlan &pl, const std::vector<std::complex<double>> &tw)
{
    const int n = pl.n;
    std::vector<double> r(n, 1.0), c(n, 1.0), nx(n);
    std::vector<double> b2[17];
    butterfly_sq<2>(b2[2]);
    butterfly_sq<3>(b2[3]);
    butterfly_sq<4>(b2[4]);
    butterfly_sq<8>(b2[8]);
    butterfly_sq<16>(b2[16]);
    auto w2 = [&](int s, int k, int j) {
        if (k == 0) return 1.0;
        const std::complex<double> w = tw[(size_t)pl.twoff[s] + (size_t)(k - 1) * (pl.len[s] / pl.radix[s]) + j];
        const double a = (double)(float)w.real(), b = (double)(float)w.imag();
        return a * a + b * b;
    };
    // forward (decimation in frequency): butterfly, then the twiddle of output k
    for (int s = 0; s < pl.ns; s++) {
        const int R = pl.radix[s], L = pl.len[s], q = L / R;
        const std::vector<double> &B = b2[R];
        for (int g0 = 0; g0 < n; g0 += L)
            for (int j = 0; j < q; j++)
                for (int k = 0; k < R; k++) {
                    double v = 0;
                    for (int m = 0; m < R; m++) v += B[(size_t)k * R + m] * r[g0 + m * q + j];
                    nx[g0 + k * q + j] = v * w2(s, k, j);
                }
        r.swap(nx);
    }
    // inverse (decimation in time, stages last to first: twiddle of input m, then the
    // butterfly); its column norms come from the transposed network, stages first to last
    for (int s = 0; s < pl.ns; s++) {
        const int R = pl.radix[s], L = pl.len[s], q = L / R;
        const std::vector<double> &B = b2[R];
        for (int g0 = 0; g0 < n; g0 += L)
            for (int j = 0; j < q; j++)
                for (int m = 0; m < R; m++) {
                    double v = 0;
                    for (int k = 0; k < R; k++) v += B[(size_t)k * R + m] * c[g0 + k * q + j];
                    nx[g0 + m * q + j] = v * w2(s, m, j);
                }
        c.swap(nx);
    }
    std::vector<double> comp(n);
    for (int p = 0; p < n; p++) comp[p] = n / std::sqrt(r[p] * c[p]);
    return comp;
}

inline void scale_table(std::vector<std::complex<double>> &tab, const std::vector<double> &comp)
{
    for (size_t k = 0; k < tab.size(); k++) tab[k] *= comp[k];
}

}  // namespace opo
