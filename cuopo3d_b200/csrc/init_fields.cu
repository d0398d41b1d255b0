// Device-side initial fields: the pump of EFields::setPumpField (EFields3D.cuh:72-137,
// 244-296) and the seeded signal noise that replaces EFields::noiseGenerator
// (EFields3D.cuh:300-315), computed on the GPU in FP64 and stored in the solver's
// precision, so that admitting an instance costs no host computation or host-to-device
// copy.  The noise is the same sequence of integer and IEEE double operations as
// opo_noise on the host, hence bit-identical to it; the pump agrees with
// opo_pump_field to the last bits of the device exp/sin/cos.

#include <cmath>

#include "solver_internal.h"

namespace {

struct PumpSpec {
    int nx, ny, nt, mode;
    double dx, dy, uX, uY, w02, T;
    double Ap0, Ap0s, tau, ts;
    double mxr, mxi;  // MX = 1 - i eta
};

__device__ __forceinline__ double noise_component(unsigned long long seed, unsigned long long idx)
{
    double acc = 0;
    for (int j = 0; j < 12; j++) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (12ull * idx + j + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        acc += (double)(z >> 11) * 0x1.0p-53;
    }
    return acc;
}

template <typename C> __device__ __forceinline__ C store(double re, double im);
template <> __device__ __forceinline__ float2 store<float2>(double re, double im) { return make_float2((float)re, (float)im); }
template <> __device__ __forceinline__ double2 store<double2>(double re, double im) { return make_double2(re, im); }

template <typename C>
__global__ void init_fields_kernel(PumpSpec ps, C *Api, C *Ap, C *As, C *Ai, unsigned long long seed, double sigma,
                                   int idler_copy)
{
    const size_t V = (size_t)ps.nx * ps.ny * ps.nt;
    for (size_t v = (size_t)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(v % ps.nx), y = (int)((v / ps.nx) % ps.ny), it = (int)(v / ((size_t)ps.nx * ps.ny));
        const double t = -ps.T * 0.5 + it * (ps.T * 0.5 - (-ps.T * 0.5)) / (ps.nt - 1);
        const double rx = (x - ps.uX) * ps.dx, ry = (y - ps.uY) * ps.dy, r2 = rx * rx + ry * ry;
        // focused profile (Ap0 / MX) exp(-r^2 / (w0^2 MX))
        const double den = ps.mxr * ps.mxr + ps.mxi * ps.mxi;
        const double ar = -r2 / ps.w02 * ps.mxr / den, ai = r2 / ps.w02 * ps.mxi / den;
        const double ea = exp(ar);
        const double fr0 = ps.Ap0 * ps.mxr / den, fi0 = -ps.Ap0 * ps.mxi / den;
        const double cr = ea * cos(ai), ci = ea * sin(ai);
        const double focr = fr0 * cr - fi0 * ci, foci = fr0 * ci + fi0 * cr;
        const double tn = t / ps.tau;
        double re = 0, im = 0;
        switch (ps.mode) {
        case OPO_PUMP_WAVEPLANE_CW: re = ps.Ap0 * exp(-r2 / ps.w02); break;
        case OPO_PUMP_WAVEPLANE_PULSED: re = ps.Ap0 * exp(-tn * tn - r2 / ps.w02); break;
        case OPO_PUMP_FOCUSED_CW: re = focr; im = foci; break;
        case OPO_PUMP_FOCUSED_PULSED: {
            const double g = exp(-tn * tn);
            re = focr * g;
            im = foci * g;
            break;
        }
        case OPO_PUMP_FOCUSED_SECH2: {
            const double g = (ps.Ap0s / ps.Ap0) / cosh(t / ps.ts);
            re = focr * g;
            im = foci * g;
            break;
        }
        case OPO_PUMP_WAVEPLANE_SECH2: re = ps.Ap0s * exp(-r2 / ps.w02) / cosh(t / ps.ts); break;
        default: break;
        }
        const C pump = store<C>(re, im);
        Api[v] = pump;
        Ap[v] = pump;
        const C s = store<C>(sigma * (noise_component(seed, 2 * v) - 6.0), sigma * (noise_component(seed, 2 * v + 1) - 6.0));
        As[v] = s;
        Ai[v] = idler_copy ? s : store<C>(0.0, 0.0);
    }
}

}  // namespace

namespace opo {

// Fills Api, Ap, As, Ai of solver s (precision prec) on `stream`.
int init_fields_device(OpoSolver *s, const OpoConfig *cfg, unsigned long long seed, double sigma, int idler_copy,
                       cudaStream_t stream)
{
    OpoParams p;
    double sc[OPO_N_SCALARS];
    int rc = opo_params_from_config(cfg, &p, sc);
    if (rc) return rc;
    const OpoParams &sp = solver_params(s);
    if (p.nx != sp.nx || p.ny != sp.ny || p.nt != sp.nt || cfg->precision != sp.precision)
        return solver_fail(s, OPO_ERR_INVALID, "init_fields: configuration does not match the solver's grid");
    if (cfg->pump_mode < OPO_PUMP_WAVEPLANE_CW || cfg->pump_mode > OPO_PUMP_WAVEPLANE_SECH2)
        return solver_fail(s, OPO_ERR_INVALID, "init_fields: unknown pump mode");
    const double kPi = 3.14159265358979323846, kC = 299792458 * 1E6 / 1E12, kEps0 = 8.8541878128E-12 * 1E12 / 1E6;
    PumpSpec ps{};
    ps.nx = p.nx; ps.ny = p.ny; ps.nt = p.nt; ps.mode = cfg->pump_mode;
    ps.dx = p.dx; ps.dy = p.dy; ps.uX = 0.5 * p.nx; ps.uY = 0.5 * p.ny;
    ps.w02 = cfg->w0 * cfg->w0;
    ps.T = p.t_window;
    const double np_ = sc[0];
    // EFields3D.cuh:247-253
    ps.tau = cfg->FWHM * std::sqrt(2.0) / (2 * std::sqrt(2 * std::log(2.0)));
    const double zR = kPi * np_ * ps.w02 / cfg->lp;
    const double eta = cfg->focal / zR;
    // 3-D peak 4P/(pi w0^2) (EFields3D.cuh:249); plane-wave 1-D 2P/(pi w0^2) (EFields1D.cuh:145-148)
    const bool one_d = p.nx == 1 && p.ny == 1;
    if (one_d && (cfg->pump_mode == OPO_PUMP_FOCUSED_CW || cfg->pump_mode == OPO_PUMP_FOCUSED_PULSED ||
                  cfg->pump_mode == OPO_PUMP_FOCUSED_SECH2))
        return solver_fail(s, OPO_ERR_INVALID, "init_fields: the 1-D solver has no focused pump");
    const double pk = one_d ? 2.0 : 4.0;
    ps.Ap0 = std::sqrt(pk * cfg->P / (kEps0 * kC * kPi * np_ * ps.w02));
    ps.ts = cfg->FWHM / (2 * std::acosh(std::sqrt(2.0)));
    ps.Ap0s = std::sqrt(pk * (cfg->P * p.t_window / (2 * ps.ts)) / (kEps0 * kC * kPi * np_ * ps.w02));
    ps.mxr = 1;
    ps.mxi = -eta;
    const size_t V = (size_t)p.nx * p.ny * p.nt;
    int blocks = (int)((V + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (sp.precision == OPO_FP64)
        init_fields_kernel<double2><<<blocks, 256, 0, stream>>>(
            ps, (double2 *)solver_field(s, 0), (double2 *)solver_field(s, 1), (double2 *)solver_field(s, 2),
            (double2 *)solver_field(s, 3), seed, sigma, idler_copy);
    else
        init_fields_kernel<float2><<<blocks, 256, 0, stream>>>(
            ps, (float2 *)solver_field(s, 0), (float2 *)solver_field(s, 1), (float2 *)solver_field(s, 2),
            (float2 *)solver_field(s, 3), seed, sigma, idler_copy);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return solver_fail(s, OPO_ERR_CUDA, cudaGetErrorString(e));
    return OPO_OK;
}

}  // namespace opo
