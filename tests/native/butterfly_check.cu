// Host-side check of the register butterflies in cuopo3d_b200/csrc/fft_radix.cuh against
// the DFT definition (compiled and run by tests/test_butterflies.py; no GPU needed).
#include <cmath>
#include <cstdio>
#include "../../cuopo3d_b200/csrc/fft_radix.cuh"

template <int R, int S, typename C> static double check()
{
    double worst = 0;
    for (int trial = 0; trial < 4; trial++) {
        C x[R], y[R];
        for (int m = 0; m < R; m++) {
            x[m].x = std::sin(1.3 * m + 0.7 * trial) + 0.1 * m;
            x[m].y = std::cos(0.9 * m * m + trial);
            y[m] = x[m];
        }
        opo::dft<R, S>(y);
        for (int k = 0; k < R; k++) {
            double re = 0, im = 0;
            for (int m = 0; m < R; m++) {
                const double a = S * 2.0 * 3.14159265358979323846 * m * k / R;
                re += x[m].x * std::cos(a) - x[m].y * std::sin(a);
                im += x[m].x * std::sin(a) + x[m].y * std::cos(a);
            }
            const double e = std::hypot(re - y[k].x, im - y[k].y);
            if (e > worst) worst = e;
        }
    }
    return worst;
}

int main()
{
    double w64 = 0, w32 = 0;
#define C64(R) { double e = check<R, 1, double2>(); if (e > w64) w64 = e; e = check<R, -1, double2>(); if (e > w64) w64 = e; }
#define C32(R) { double e = check<R, 1, float2>(); if (e > w32) w32 = e; e = check<R, -1, float2>(); if (e > w32) w32 = e; }
    C64(2) C64(3) C64(4) C64(8) C64(16)
    C32(2) C32(3) C32(4) C32(8) C32(16)
    std::printf("max_err_fp64 %.3e max_err_fp32 %.3e\n", w64, w32);
    return (w64 < 1e-13 && w32 < 1e-5) ? 0 : 1;
}
