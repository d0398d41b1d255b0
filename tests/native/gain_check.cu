// Host-side check of the FP32 transform-pair gain compensation (cuopo3d_b200/csrc/
// fft_gain.h), compiled and run by tests/test_butterflies.py; no GPU needed.
//
// For each plan, the forward (decimation in frequency) and inverse (decimation in time)
// transforms are built as dense operators in FP64 arithmetic with the FP32 kernels'
// constants: the butterflies' matrices from dft<R> on float2 unit vectors and the stage
// twiddles rounded to FP32.  The squared row norms of the forward operator and column
// norms of the inverse, summed by brute force, must equal the squared-magnitude network
// of fp32_pair_compensation; and the compensated pair with a unit-modulus table must
// preserve the energy of random white inputs to rounding, where the uncompensated one
// drains it.
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "../../cuopo3d_b200/csrc/fft_gain.h"

using cd = std::complex<double>;

static const double kPi = 3.14159265358979323846;

// Plan from a radix list (AxisPlan layout, as the solver builds it).
static opo::AxisPlan make_plan(const std::vector<int> &rad, std::vector<cd> &tw)
{
    opo::AxisPlan p{};
    int n = 1;
    for (int r : rad) n *= r;
    p.n = n;
    p.ns = (int)rad.size();
    int L = n;
    for (int s = 0; s < p.ns; s++) {
        const int R = rad[s], q = L / R;
        p.radix[s] = R;
        p.len[s] = L;
        p.twoff[s] = (int)tw.size();
        p.q[s].d = (unsigned)q;
        for (int k = 1; k < R; k++)
            for (int j = 0; j < q; j++) tw.push_back(std::polar(1.0, -2 * kPi * (double)j * k / L));
        L = q;
    }
    return p;
}

template <int R> static void butterfly_matrix(int S, std::vector<cd> &B)
{
    B.assign((size_t)R * R, cd(0, 0));
    for (int m = 0; m < R; m++) {
        float2 x[R];
        for (int k = 0; k < R; k++) x[k] = make_float2(k == m ? 1.f : 0.f, 0.f);
        if (S > 0)
            opo::dft<R, +1>(x);
        else
            opo::dft<R, -1>(x);
        for (int k = 0; k < R; k++) B[(size_t)k * R + m] = cd(x[k].x, x[k].y);
    }
}

static void butterfly(int R, int S, std::vector<cd> &B)
{
    switch (R) {
    case 2: butterfly_matrix<2>(S, B); break;
    case 3: butterfly_matrix<3>(S, B); break;
    case 4: butterfly_matrix<4>(S, B); break;
    case 8: butterfly_matrix<8>(S, B); break;
    default: butterfly_matrix<16>(S, B); break;
    }
}

static cd tw32(const opo::AxisPlan &p, const std::vector<cd> &tw, int s, int k, int j)
{
    if (k == 0) return cd(1, 0);
    const cd w = tw[(size_t)p.twoff[s] + (size_t)(k - 1) * (p.len[s] / p.radix[s]) + j];
    return cd((float)w.real(), (float)w.imag());
}

// Forward transform (sign -1, twiddle multiplies by w) of x in place.
static void forward(const opo::AxisPlan &p, const std::vector<cd> &tw, std::vector<cd> &x)
{
    const int n = p.n;
    std::vector<cd> y(n), B;
    for (int s = 0; s < p.ns; s++) {
        const int R = p.radix[s], L = p.len[s], q = L / R;
        butterfly(R, -1, B);
        for (int g0 = 0; g0 < n; g0 += L)
            for (int j = 0; j < q; j++)
                for (int k = 0; k < R; k++) {
                    cd v = 0;
                    for (int m = 0; m < R; m++) v += B[(size_t)k * R + m] * x[g0 + m * q + j];
                    y[g0 + k * q + j] = v * tw32(p, tw, s, k, j);
                }
        x.swap(y);
    }
}

// Inverse transform (sign +1, twiddle multiplies by conj(w)) of x in place.
static void inverse(const opo::AxisPlan &p, const std::vector<cd> &tw, std::vector<cd> &x)
{
    const int n = p.n;
    std::vector<cd> y(n), B;
    for (int s = p.ns - 1; s >= 0; s--) {
        const int R = p.radix[s], L = p.len[s], q = L / R;
        butterfly(R, +1, B);
        for (int g0 = 0; g0 < n; g0 += L)
            for (int j = 0; j < q; j++) {
                cd in[16];
                for (int m = 0; m < R; m++) in[m] = x[g0 + m * q + j] * std::conj(tw32(p, tw, s, m, j));
                for (int k = 0; k < R; k++) {
                    cd v = 0;
                    for (int m = 0; m < R; m++) v += B[(size_t)k * R + m] * in[m];
                    y[g0 + k * q + j] = v;
                }
            }
        x.swap(y);
    }
}

int main()
{
    const std::vector<std::vector<int>> plans = {{8, 8, 4}, {16, 8}, {8, 16}, {16, 16}, {4, 3, 4, 2}, {8, 3, 8},
                                                 {16, 3, 4}, {4, 16, 16}, {8, 3, 3, 4}};
    int bad = 0;
    std::mt19937_64 rng(7);
    std::normal_distribution<double> nd;
    for (const auto &rad : plans) {
        std::vector<cd> tw;
        const opo::AxisPlan p = make_plan(rad, tw);
        const int n = p.n;
        const std::vector<double> comp = opo::fp32_pair_compensation(p, tw);
        // brute force: rows of the forward operator, columns of the inverse
        std::vector<double> r(n, 0.0), c(n, 0.0);
        for (int i = 0; i < n; i++) {
            std::vector<cd> e(n, cd(0, 0));
            e[i] = 1;
            forward(p, tw, e);
            for (int q = 0; q < n; q++) r[q] += std::norm(e[q]);
            std::vector<cd> u(n, cd(0, 0));
            u[i] = 1;
            inverse(p, tw, u);
            for (int q = 0; q < n; q++) c[i] += std::norm(u[q]);
        }
        double worst = 0, dev = 0;
        for (int q = 0; q < n; q++) {
            const double want = n / std::sqrt(r[q] * c[q]);
            worst = std::max(worst, std::abs(comp[q] / want - 1));
            dev = std::max(dev, std::abs(comp[q] - 1));
        }
        // energy gain of the pair with a unit-modulus table (1/n normalisation), white inputs
        double g_plain = 0, g_comp = 0, e_in = 0;
        for (int trial = 0; trial < 64; trial++) {
            std::vector<cd> x(n);
            for (auto &v : x) v = cd(nd(rng), nd(rng));
            std::vector<cd> a = x, b;
            forward(p, tw, a);
            b = a;
            for (int q = 0; q < n; q++) {
                const cd t = std::polar(1.0, 0.37 * q * q) / (double)n;
                a[q] *= t;
                b[q] *= t * comp[q];
            }
            inverse(p, tw, a);
            inverse(p, tw, b);
            for (int q = 0; q < n; q++) {
                e_in += std::norm(x[q]);
                g_plain += std::norm(a[q]);
                g_comp += std::norm(b[q]);
            }
        }
        const double d_plain = g_plain / e_in - 1, d_comp = g_comp / e_in - 1;
        const bool ok = worst < 1e-13 && dev > 1e-9 && dev < 1e-6 && std::abs(d_comp) < 0.2 * std::abs(d_plain);
        std::printf("plan n=%4d ns=%d: network vs brute force %.2e, |comp-1| max %.2e, energy gain "
                    "plain %+.3e compensated %+.3e %s\n",
                    n, p.ns, worst, dev, d_plain, d_comp, ok ? "ok" : "FAIL");
        bad += !ok;
    }
    return bad ? 1 : 0;
}
