// Test infrastructure, NOT product code: FP64 CPU restatement of the cuOPO3D
// split-step solver.  See opo_oracle.h for the contract.  Citations are
// file:line in alfredos84/cuOPO3D (src/...).
//
// Parity status: pinned by tests/golden (outputs of the reference's own code built by
// oracle/refharness and run on a B200).

#include "opo_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

namespace {

// Physical constants, src/headers/DtypesConsts.cuh:55-57.
const double PI = 3.14159265358979323846;
const double C = 299792458 * 1E6 / 1E12;        // um/ps
const double EPS0 = 8.8541878128E-12 * 1E12 / 1E6; // W ps / (V^2 um)

// ---------------------------------------------------------------------------------
// Crystal Sellmeier models.

// PPLN extraordinary index, src/headers/CrystalsBase/PPLN.cuh:97-117 (Jundt).
struct PPLNModel {
    double a1 = 5.35583, a2 = 0.100473, a3 = 0.20692, a4 = 100.0, a5 = 11.34927,
           a6 = 1.5334e-2, b1 = 4.629e-7, b2 = 3.862e-8, b3 = -0.89e-8, b4 = 2.657e-5;
    double G1, G2, G3, G4;
    explicit PPLNModel(double T) { init(T); }
    void init(double T)
    {
        double f = (T - 24.5) * (T + 570.82);
        G1 = a1 + b1 * f; G2 = a2 + b2 * f; G3 = a3 + b3 * f; G4 = a4 + b4 * f;
    }
    double n(double L) const
    {
        return std::sqrt(G1 + G2 / (L * L - G3 * G3) + G4 / (L * L - a5 * a5) - a6 * L * L);
    }
    // PPLN.cuh:122-143
    double res(double L, int p) const
    {
        return G2 / std::pow(L * L - G3 * G3, p) + G4 / std::pow(L * L - a5 * a5, p);
    }
    double res2c(double L) const { return res(L, 2) + a6; }  // (resonances(2) + a6)
};

// MgO:PPLN extraordinary index, src/headers/CrystalsBase/MgOPPLN.cuh:97-143 (Gayer): the
// PPLN form with other coefficients.
struct MgOPPLNModel : PPLNModel {
    explicit MgOPPLNModel(double T) : PPLNModel(T)
    {
        a1 = 5.756; a2 = 0.0983; a3 = 0.2020; a4 = 189.32; a5 = 12.52; a6 = 1.32e-2;
        b1 = 2.860e-6; b2 = 4.700e-8; b3 = 6.113e-8; b4 = 1.516e-4;
        init(T);
    }
};

// MgO:sPPLT index, src/headers/CrystalsBase/MgOsPPLT.cuh:96-132 (Bruner).
struct SPPLTModel {
    double A = 4.502483, B = 0.007294, Cc = 0.185087, D = -0.02357, E = 0.073423,
           F = 0.199595, G = 0.001, H = 7.99724;
    double b, c;
    explicit SPPLTModel(double T)
    {
        b = 3.483933e-8 * std::pow(T + 273.15, 2);
        c = 1.607839e-8 * std::pow(T + 273.15, 2);
    }
    double n(double L) const
    {
        return std::sqrt(A + (B + b) / (L * L - (Cc + c) * (Cc + c)) + E / (L * L - F * F) +
                         G / (L * L - H * H) + D * L * L);
    }
    double res(double L, int p) const
    {
        return (B + b) / std::pow(L * L - (Cc + c) * (Cc + c), p) +
               E / std::pow(L * L - F * F, p) + G / std::pow(L * L - H * H, p);
    }
    double res2c(double L) const { return res(L, 2) - D; }  // (resonances(2) - D)
};

// Derivatives shared by both models (PPLN.cuh:149-259, MgOsPPLT.cuh:138-226): with
// R2 = the model's "resonances(2) +/- constant" term,
//   dn/dl   = -L R2 / n
//   d2n/dl2 = (L dn/dl / n^2 - 1/n) R2 + 4 L^2 / n res3
//   d3n/dl3 = ((2 dn + L d2n)/n^2 - 2 L dn^2/n^3) R2 + (12 L/n - 4 L^2/n d2n (1-1/n)) res3
//             - 24 L^3 / n res4
//   vg = c / (n - L dn/dl);  b2 = L^3 d2n / (2 pi c^2);
//   b3 = -L^4 / (4 pi^2 c^3) (3 d2n + L d3n)
template <class M> struct Dispersive {
    M m;
    explicit Dispersive(double T) : m(T) {}
    double n(double L) const { return m.n(L); }
    double dn(double L) const { return -L * m.res2c(L) / m.n(L); }
    double d2n(double L) const
    {
        double nn = m.n(L);
        return (L * dn(L) / (nn * nn) - 1 / nn) * m.res2c(L) + 4 * L * L / nn * m.res(L, 3);
    }
    double d3n(double L) const
    {
        double nn = m.n(L), d1 = dn(L), d2 = d2n(L);
        double A1 = (2 * d1 + L * d2) / (nn * nn);
        double A2 = -2 * L * d1 * d1 / (nn * nn * nn);
        double AA = (A1 + A2) * m.res2c(L);
        double B1 = 12 * L / nn;
        double B2 = -4 * L * L / nn * d2 * (1 - 1 / nn);
        double BB = (B1 + B2) * m.res(L, 3);
        double CC = -24 * L * L * L / nn * m.res(L, 4);
        return AA + BB + CC;
    }
    double GV(double L) const { return C / (n(L) - L * dn(L)); }
    double GVD(double L) const { return std::pow(L, 3) * d2n(L) / (2 * PI * C * C); }
    double TOD(double L) const
    {
        return -std::pow(L, 4) / (4 * PI * PI * C * C * C) * (3 * d2n(L) + L * d3n(L));
    }
    // the exact TOD: d3n from a central difference of d2n (the reference's d3ndl3 is
    // not the third derivative; it only prints that TOD)
    double TODexact(double L) const
    {
        const double h = 1e-4 * L;
        const double d3 = (d2n(L - 2 * h) - 8 * d2n(L - h) + 8 * d2n(L + h) - d2n(L + 2 * h)) / (12 * h);
        return -std::pow(L, 4) / (4 * PI * PI * C * C * C) * (3 * d2n(L) + L * d3);
    }
};

// ZGP ordinary / extraordinary index, src/headers/CrystalsBase/ZGP.cuh:103-226 (Zelmon):
//   n^2 = A + B L^2/(L^2 - CC) + D L^2/(L^2 - E),  fb_p = B L^2/(L^2-CC)^p, fd_p likewise,
//   dn/dl = -(CC fb_2 + E fd_2) / (n L),
//   d2n/dl2 = (CC fb_3 (CC/L^2 + 3) + E fd_3 (E/L^2 + 3) - (dn/dl)^2) / n.
// The reference has no third derivative for ZGP; TOD here differentiates d2n/dl2
// numerically (central difference), independently of the library's closed form.
struct ZGPModel {
    double A, B, CC, D, E;
    explicit ZGPModel(bool e)
    {
        if (e) { A = 8.0929; B = 1.8649; CC = 0.41468; D = 0.84052; E = 452.05; }
        else { A = 8.0409; B = 1.68625; CC = 0.40824; D = 1.2880; E = 611.05; }
    }
    double n(double L) const { return std::sqrt(A + B * L * L / (L * L - CC) + D * L * L / (L * L - E)); }
    double fb(double L, int p) const { return B * L * L / std::pow(L * L - CC, p); }
    double fd(double L, int p) const { return D * L * L / std::pow(L * L - E, p); }
    double dn(double L) const { return -(CC * fb(L, 2) + E * fd(L, 2)) / (n(L) * L); }
    double d2n(double L) const
    {
        const double d1 = dn(L);
        return (CC * fb(L, 3) * (CC / (L * L) + 3) + E * fd(L, 3) * (E / (L * L) + 3) - d1 * d1) / n(L);
    }
    double d3n(double L) const
    {
        const double h = 1e-4 * L;
        return (d2n(L - 2 * h) - 8 * d2n(L - h) + 8 * d2n(L + h) - d2n(L + 2 * h)) / (12 * h);
    }
    double GV(double L) const { return C / (n(L) - L * dn(L)); }
    double GVD(double L) const { return std::pow(L, 3) * d2n(L) / (2 * PI * C * C); }
    double TOD(double L) const
    {
        return -std::pow(L, 4) / (4 * PI * PI * C * C * C) * (3 * d2n(L) + L * d3n(L));
    }
    double TODexact(double L) const { return TOD(L); }
};

// n, vg, b2, b3 (as the reference prints it) and the exact b3 of one index of a crystal
// (0: ok, -2: unknown crystal).
int crystalIndex(int crystal, double T, bool extraordinary, double L, double out[5])
{
    auto fill = [&](const auto &m) {
        out[0] = m.n(L); out[1] = m.GV(L); out[2] = m.GVD(L); out[3] = m.TOD(L); out[4] = m.TODexact(L);
    };
    switch (crystal) {
    case OR_PPLN: fill(Dispersive<PPLNModel>(T)); return 0;
    case OR_MGOSPPLT: fill(Dispersive<SPPLTModel>(T)); return 0;
    case OR_MGOPPLN: fill(Dispersive<MgOPPLNModel>(T)); return 0;
    case OR_ZGP: fill(ZGPModel(extraordinary)); return 0;
    default: return -2;
    }
}

// ---------------------------------------------------------------------------------
// FFT: mixed-radix (factors 4, 2, 3, 5, then any prime) decimation in time, written
// from the DFT definition X[k] = sum_j x[j] exp(sign 2 pi i j k / n), unnormalised.
// sign = -1 is cuFFT's FORWARD, +1 its INVERSE.

struct FFTPlan {
    int n = 0;
    std::vector<int> factors;
    std::vector<cd> w;  // exp(-2 pi i k / n)
    explicit FFTPlan(int n_) : n(n_)
    {
        int m = n;
        for (int r : {4, 2, 3, 5}) {
            while (m % r == 0) { factors.push_back(r); m /= r; }
        }
        for (int r = 7; m > 1; r += 2)
            while (m % r == 0) { factors.push_back(r); m /= r; }
        w.resize(n);
        for (int k = 0; k < n; k++) w[k] = std::polar(1.0, -2 * PI * k / n);
    }
};

void fftRec(const FFTPlan &P, int sign, const cd *in, cd *out, int n, int stride, int fi,
            int twStride, cd *scratch)
{
    if (n == 1) { out[0] = in[0]; return; }
    int r = P.factors[fi], m = n / r;
    for (int q = 0; q < r; q++)
        fftRec(P, sign, in + (size_t)q * stride, out + (size_t)q * m, m, stride * r, fi + 1,
               twStride * r, scratch);
    cd t[64];
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < r; q++) {
            cd tw = P.w[((size_t)q * k * twStride) % P.n];
            if (sign > 0) tw = std::conj(tw);
            t[q] = out[(size_t)q * m + k] * tw;
        }
        for (int s = 0; s < r; s++) {
            cd acc = 0;
            for (int q = 0; q < r; q++) {
                cd wr = P.w[((size_t)q * s * (P.n / r)) % P.n];
                if (sign > 0) wr = std::conj(wr);
                acc += t[q] * wr;
            }
            scratch[s] = acc;
        }
        for (int s = 0; s < r; s++) out[(size_t)s * m + k] = scratch[s];
    }
}

struct FFTCache {
    std::vector<FFTPlan *> plans;
    ~FFTCache()
    {
        for (auto *p : plans) delete p;
    }
    const FFTPlan &get(int n)
    {
        for (auto *p : plans)
            if (p->n == n) return *p;
        plans.push_back(new FFTPlan(n));
        return *plans.back();
    }
};

// Transform x (length n) in place; tmp must hold n values.
void fft1(const FFTPlan &P, int sign, cd *x, cd *tmp)
{
    cd scratch[64];
    std::memcpy((void *)tmp, (void *)x, sizeof(cd) * P.n);
    fftRec(P, sign, tmp, x, P.n, 1, 0, 1, scratch);
}

// ---------------------------------------------------------------------------------
// Complex exponentials as the reference writes them (Operators.cuh:166-182).
inline cd cpxExp(double a) { return cd(std::cos(a), std::sin(a)); }
inline cd cpxExp(cd a) { return cd(std::exp(a.real()) * std::cos(a.imag()), std::exp(a.real()) * std::sin(a.imag())); }
// real / complex, Operators.cuh:136-144
inline cd realDiv(double a, cd b)
{
    double den = b.real() * b.real() + b.imag() * b.imag();
    return cd(a * b.real() / den, -a * b.imag() / den);
}

size_t idx3(const OrParams *p, int x, int y, int t)
{
    return (size_t)t * p->nx * p->ny + (size_t)y * p->nx + x;  // Common.cuh:167-170
}

// ---------------------------------------------------------------------------------
// Nonlinear step.  Coupled-wave right-hand side, Solver3D.cuh:365-382:
//   dAp = i kp As Ai e^{-i dk z},  dAs = i ks Ap Ai* e^{+i dk z},  dAi = i ki Ap As* e^{+i dk z}
// The shipped code multiplies dk z by 0 (OR_PHYSICS restores it).
inline void rhs(const OrParams *p, double z, const cd &Ap, const cd &As, const cd &Ai, cd &dp,
                cd &ds, cd &di)
{
    const cd I(0, 1);
    dp = I * p->kappa[0] * As * Ai;
    ds = I * p->kappa[1] * Ap * std::conj(Ai);
    di = I * p->kappa[2] * Ap * std::conj(As);
    if (p->flags & OR_PHYSICS) {
        cd ph = cpxExp(p->dk * z);
        dp *= std::conj(ph);
        ds *= ph;
        di *= ph;
    }
}

// One RK4 step of size s = dz/2 over every voxel, Solver3D.cuh:872-943 with the
// kernels at :386-425.  Shipped stage arguments are A + 0.5 k1, A + 0.5 k2, A + k3
// (no step size); OR_PHYSICS uses A + (s/2) k1, A + (s/2) k2, A + s k3.
void rk4Half(const OrParams *p, double z, cd *Ap, cd *As, cd *Ai)
{
    const size_t V = (size_t)p->nx * p->ny * p->nt;
    const double s = 0.5 * p->dz;
    const bool phys = (p->flags & OR_PHYSICS) != 0;
    const double c1 = phys ? 0.5 * s : 0.5, c3 = phys ? s : 1.0;
    // Stage positions (Solver3D.cuh:911-929): z, z + dz/4, z + dz/4, z + dz/2.
    const double z1 = z, z2 = z + p->dz / 4.0, z4 = z + p->dz / 2.0;
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < (long long)V; v++) {
        cd p0 = Ap[v], s0 = As[v], i0 = Ai[v];
        cd k1p, k1s, k1i, k2p, k2s, k2i, k3p, k3s, k3i, k4p, k4s, k4i;
        rhs(p, z1, p0, s0, i0, k1p, k1s, k1i);
        rhs(p, z2, p0 + k1p * c1, s0 + k1s * c1, i0 + k1i * c1, k2p, k2s, k2i);
        rhs(p, z2, p0 + k2p * c1, s0 + k2s * c1, i0 + k2i * c1, k3p, k3s, k3i);
        rhs(p, z4, p0 + k3p * c3, s0 + k3s * c3, i0 + k3i * c3, k4p, k4s, k4i);
        Ap[v] = p0 + (k1p + 2.0 * k2p + 2.0 * k3p + k4p) * s / 6.0;
        As[v] = s0 + (k1s + 2.0 * k2s + 2.0 * k3s + k4s) * s / 6.0;
        Ai[v] = i0 + (k1i + 2.0 * k2i + 2.0 * k3i + k4i) * s / 6.0;
    }
}

// ---------------------------------------------------------------------------------
// Linear steps.

// Dispersion propagators, Solver3D.cuh:153-169:
//   eiLz_f(w) = exp(i dz w (vinv_f + w b2_f / 2)) exp(-alpha_f dz / 2)
// (OR_TOD, not in the reference: the phase gains dz w^3 b3_f / 6).
void dispersionTable(const OrParams *p, const double *w, int f, double len, bool absorb,
                     std::vector<cd> &tab)
{
    tab.resize(p->nt);
    const double b3 = (p->flags & OR_TOD) ? p->beta3[f] : 0.0;
    for (int k = 0; k < p->nt; k++) {
        tab[k] = cpxExp(len * w[k] * (p->vinv[f] + 0.5 * w[k] * p->beta2[f] + w[k] * w[k] * b3 / 6.0));
        if (absorb) tab[k] *= std::exp(-0.5 * p->alpha[f] * len);
    }
}

// t-axis operator on selected fields: per pixel line, INVERSE transform, times
// tab/NT, FORWARD transform (Solver3D.cuh:572-639 with the launch grid and the 1/NT
// scale corrected).  With OR_ASIS_Q2 only pixels on row y=0 are transformed and the
// scale is 1/(NX NY NT), as the shipped <<<64,64>>> launches do.
void tAxisOp(const OrParams *p, FFTCache &cache, cd *F[3], const std::vector<cd> tab[3],
             unsigned mask)
{
    const int nx = p->nx, ny = p->ny, nt = p->nt;
    const FFTPlan &P = cache.get(nt);
    const bool q2 = (p->flags & OR_ASIS_Q2) != 0;
    const double scale = q2 ? 1.0 / ((double)nx * ny * nt) : 1.0 / nt;
    const int npix = q2 ? nx : nx * ny;
#pragma omp parallel
    {
        std::vector<cd> line(nt), tmp(nt);
#pragma omp for schedule(static)
        for (int pix = 0; pix < npix; pix++) {
            int x = pix % nx, y = pix / nx;
            for (int f = 0; f < 3; f++) {
                if (!(mask & (1u << f))) continue;
                for (int t = 0; t < nt; t++) line[t] = F[f][idx3(p, x, y, t)];
                fft1(P, +1, line.data(), tmp.data());
                for (int t = 0; t < nt; t++) line[t] *= scale * tab[f][t];
                fft1(P, -1, line.data(), tmp.data());
                for (int t = 0; t < nt; t++) F[f][idx3(p, x, y, t)] = line[t];
            }
        }
    }
}

// Diffraction propagator on the centred grid then fftshift-ed, Solver3D.cuh:282-301
// and EFields3D.cuh:141-171,332-351:
//   eiQz(x,y) = exp(sign len 2 pi^2 / k (dfX^2 (x-NX/2)^2 + dfY^2 (y-NY/2)^2)) [exp(-alpha len/2)]
// with dfX = 1/(dx NX).  After the 2-D shift the value at FFT bin (i, j) is the
// centred value at ((i + NX/2) mod NX, (j + NY/2) mod NY).
void diffractionTable(const OrParams *p, double k, double sign, double len, double alpha,
                      std::vector<cd> &tab)
{
    const int nx = p->nx, ny = p->ny;
    const double dfX = 1 / p->dx / nx, dfY = 1 / p->dy / ny;
    const double uX = 0.5 * nx, uY = 0.5 * ny;
    std::vector<cd> centred((size_t)nx * ny);
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            double q = dfX * dfX * std::pow(x - uX, 2) + dfY * dfY * std::pow(y - uY, 2);
            cd v = cpxExp(sign * len * (2 * std::pow(PI, 2) / k * q));
            if (alpha >= 0) v *= std::exp(-0.5 * alpha * len);
            centred[(size_t)y * nx + x] = v;
        }
    tab.resize((size_t)nx * ny);
    const int cx = nx / 2, cy = ny / 2;
    for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
            int sx = (x + cx) % nx, sy = (y + cy) % ny;
            tab[(size_t)y * nx + x] = centred[(size_t)sy * nx + sx];
        }
}

// (x,y) operator on selected fields: per t-plane, 2-D FORWARD transform, times the
// table, 2-D INVERSE transform, times `scale` (Solver3D.cuh:726-788 and :818-869).
void xyOp(const OrParams *p, FFTCache &cache, cd *F[3], const std::vector<cd> tab[3],
          unsigned mask, double scale)
{
    const int nx = p->nx, ny = p->ny, nt = p->nt;
    const FFTPlan &PX = cache.get(nx);
    const FFTPlan &PY = cache.get(ny);
#pragma omp parallel
    {
        std::vector<cd> plane((size_t)nx * ny), col(ny), tmp(nx > ny ? nx : ny);
#pragma omp for schedule(static)
        for (int job = 0; job < nt * 3; job++) {
            int t = job / 3, f = job % 3;
            if (!(mask & (1u << f))) continue;
            cd *base = F[f] + (size_t)t * nx * ny;
            std::memcpy((void *)plane.data(), (void *)base, sizeof(cd) * nx * ny);
            for (int dir = -1; dir <= 1; dir += 2) {
                for (int y = 0; y < ny; y++) fft1(PX, dir, plane.data() + (size_t)y * nx, tmp.data());
                for (int x = 0; x < nx; x++) {
                    for (int y = 0; y < ny; y++) col[y] = plane[(size_t)y * nx + x];
                    fft1(PY, dir, col.data(), tmp.data());
                    for (int y = 0; y < ny; y++) plane[(size_t)y * nx + x] = col[y];
                }
                if (dir < 0)
                    for (size_t v = 0; v < (size_t)nx * ny; v++) plane[v] *= tab[f][v];
            }
            for (size_t v = 0; v < (size_t)nx * ny; v++) base[v] = plane[v] * scale;
        }
    }
}

struct Run {
    const OrParams *p;
    const double *w;
    FFTCache cache;
    std::vector<cd> dispTab[3], diffTab[3], freeTab[3], gddTab[3];

    Run(const OrParams *p_, const double *w_) : p(p_), w(w_)
    {
        const bool phys = (p->flags & OR_PHYSICS) != 0;
        for (int f = 0; f < 3; f++) {
            // Shipped code applies exp(-alpha dz/2) in both propagators (Solver3D.cuh:163-165
            // and :294-296); physics mode keeps it only in the diffraction one.
            dispersionTable(p, w, f, p->dz, !phys, dispTab[f]);
            diffractionTable(p, p->kdiff[f], -1.0, p->dz, p->alpha[f], diffTab[f]);
            // Free-space return, Solver3D.cuh:305-323 (signal and idler, no absorption).
            diffractionTable(p, p->kdiff[f], +1.0, p->free_len, -1.0, freeTab[f]);
            // GDD compensation, Solver3D.cuh:261-277 and :676: exp(i w^2 GDD / 2).
            gddTab[f].resize(p->nt);
            for (int k = 0; k < p->nt; k++) gddTab[f][k] = cpxExp(0.5 * w[k] * w[k] * p->gdd);
        }
    }

    void dispersion(cd *F[3]) { tAxisOp(p, cache, F, dispTab, 7u); }

    void diffraction(cd *F[3])
    {
        const double nxy = (double)p->nx * p->ny;
        const double scale = (p->flags & OR_ASIS_Q1) ? 1.0 / (nxy * p->nt) : 1.0 / nxy;
        xyOp(p, cache, F, diffTab, 7u, scale);
    }

    // Split-step over the crystal, Solver3D.cuh:946-960:
    //   for each z-step: RK4(dz/2), dispersion(dz), diffraction(dz), RK4(dz/2)
    void ssfm(cd *F[3])
    {
        const bool phys = (p->flags & OR_PHYSICS) != 0;
        for (int k = 0; k < p->n_steps; k++) {
            double z = k * p->dz;
            rk4Half(p, z, F[0], F[1], F[2]);
            if (p->flags & OR_DISPERSION) dispersion(F);
            if (p->flags & OR_DIFFRACTION) diffraction(F);
            rk4Half(p, phys ? z + 0.5 * p->dz : z, F[0], F[1], F[2]);
        }
    }
};

}  // namespace

extern "C" {

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Step count of `for (real_t z = 0; z <= Lcr; z += dz)`, Solver3D.cuh:949, in FP32
// (the shipped real_t) or FP64.
int or_zloop_steps(double Lcr, double dz, int f32)
{
    int n = 0;
    if (f32) {
        float L = (float)Lcr, d = (float)dz;
        for (float z = 0; z <= L; z += d) n++;
    } else {
        for (double z = 0; z <= Lcr; z += dz) n++;
    }
    return n;
}

void or_fft(int n, int sign, double *data)
{
    FFTPlan P(n);
    std::vector<cd> tmp(n);
    fft1(P, sign, reinterpret_cast<cd *>(data), tmp.data());
}

// Counter-based noise: each component is sigma * (sum of 12 uniforms - 6) with the
// uniforms from splitmix64, so every value is a fixed sequence of IEEE operations and
// identical on any host or device.  Replaces the reference's wall-clock-seeded
// std::normal_distribution (EFields3D.cuh:300-315).
void or_noise(uint64_t seed, double sigma, size_t n_complex, double *out)
{
    for (size_t v = 0; v < 2 * n_complex; v++) {
        double acc = 0;
        for (int j = 0; j < 12; j++) {
            uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(12 * v + j + 1);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z = z ^ (z >> 31);
            acc += (double)(z >> 11) * 0x1.0p-53;
        }
        out[v] = sigma * (acc - 6.0);
    }
}

void or_power_sums(int n, const double *A, double *sum_abs2)
{
    double s = 0;
    for (int v = 0; v < n; v++) s += A[2 * v] * A[2 * v] + A[2 * v + 1] * A[2 * v + 1];
    *sum_abs2 = s;
}

// Build every derived quantity of a run from its physical description:
//   crystal constructor  PPLN.cuh:51-78 / MgOsPPLT.cuh:51-78
//   EFields constructor  EFields3D.cuh:199-227 (kappa, k; Q8: kp uses ns, ki uses ls)
//   Cavity constructor   Cavity3D.cuh:42-49 (trt, dt)
//   t/w grids            EFields3D.cuh:319-328, Common.cuh:120-128, EFields3D.cuh:58-68
//   pump field           EFields3D.cuh:244-296 with the kernels at :72-137
int or_crystal_dispersion(int crystal, double T, int extraordinary, double L, double out[5])
{
    if (!out || !(L > 0)) return -1;
    return crystalIndex(crystal, T, extraordinary != 0, L, out);
}

int or_setup(const OrPhys *in, OrParams *o, double *sc, double *t, double *w, double *Api)
{
    const int nx = in->nx, ny = in->ny, nt = in->nt;
    // nx = ny = 1 without diffraction: the plane-wave 1-D solver (Solver1D.cuh)
    const bool diff = (in->flags & OR_DIFFRACTION) != 0;
    if (nx < (diff ? 2 : 1) || ny < (diff ? 2 : 1) || nt < 2 || in->nz < 2) return -1;
    const double lp = in->lp, ls = in->ls, li = ls * lp / (ls - lp);
    double n[3], v[3], b2[3], b3[3], d33, alpha[3];
    const double L3[3] = {lp, ls, li};
    double b3x[3];
    for (int f = 0; f < 3; f++) {
        double q[5];
        if (crystalIndex(in->crystal, in->T, (in->pol >> f) & 1u, L3[f], q)) return -2;
        n[f] = q[0]; v[f] = q[1]; b2[f] = q[2]; b3[f] = q[3]; b3x[f] = q[4];
    }
    // d33 and absorption: PPLN.cuh:57-60, MgOPPLN.cuh:57-60, MgOsPPLT.cuh:57-60, ZGP.cuh:55-58
    if (in->crystal == OR_PPLN || in->crystal == OR_MGOPPLN) {
        d33 = 25.20e-6;
        alpha[0] = 0.025e-4; alpha[1] = 0.002e-4; alpha[2] = 0.002e-4;
    } else {
        d33 = in->crystal == OR_ZGP ? 75.0e-6 : 11.0e-6;
        alpha[0] = 1.57e-4; alpha[1] = 0.17e-6; alpha[2] = 0.17e-6;
    }
    double dQ = 2.0 * d33 / PI;
    if (in->dQ > 0) dQ = in->dQ;
    for (int f = 0; f < 3; f++)
        if (in->alpha[f] >= 0) alpha[f] = in->alpha[f];
    const double dx = nx > 1 ? in->LX / (nx - 1.0) : 0.0, dy = ny > 1 ? in->LY / (ny - 1.0) : 0.0,
                 dz = in->Lcr / (in->nz - 1.0);
    const bool phys = (in->flags & OR_PHYSICS) != 0;
    // Wavevectors: shipped kp = 2 pi ns / lp and ki = 2 pi ni / ls (Q8).
    const double kp = phys ? 2.0 * PI * n[0] / lp : 2.0 * PI * n[1] / lp;
    const double ks = 2.0 * PI * n[1] / ls;
    const double ki = phys ? 2.0 * PI * n[2] / li : 2.0 * PI * n[2] / ls;
    // ZGP is not quasi-phase matched: no grating term (ZGP.cuh:76)
    const double dk = kp - ks - ki - (in->crystal == OR_ZGP ? 0.0 : 2.0 * PI / in->Lambda);
    const double kappa[3] = {2 * PI * dQ / (n[0] * lp), 2 * PI * dQ / (n[1] * ls),
                             2 * PI * dQ / (n[2] * li)};
    const double trt = (in->Lcav + in->Lcr * (n[1] - 1)) / C;
    const double dt = trt / (nt - 1);
    int nsteps = in->n_steps > 0 ? in->n_steps : or_zloop_steps(in->Lcr, dz, in->zloop_f32);

    o->nx = nx; o->ny = ny; o->nt = nt; o->n_steps = nsteps; o->flags = in->flags;
    o->dz = (phys && in->n_steps > 0) ? in->Lcr / in->n_steps : dz;
    o->Lcr = in->Lcr; o->dx = dx; o->dy = dy;
    for (int f = 0; f < 3; f++) {
        o->kappa[f] = kappa[f]; o->beta2[f] = b2[f]; o->beta3[f] = b3x[f]; o->alpha[f] = alpha[f];
    }
    o->kdiff[0] = kp; o->kdiff[1] = ks; o->kdiff[2] = ki;
    // Group-delay frame, Solver3D.cuh:163-165: pump 1/vp-1/vi, signal 0, idler 1/vi-1/vs.
    o->vinv[0] = 1 / v[0] - 1 / v[2];
    o->vinv[1] = 1 / v[1] - 1 / v[1];
    o->vinv[2] = 1 / v[2] - 1 / v[1];
    o->dk = dk;
    o->Rs = in->Rs; o->Ri = in->Ri; o->detuning = in->detuning;
    o->resonant = in->resonant;
    o->gdd = in->gdd_gamma != 0 ? -(in->gdd_gamma) * b2[1] * in->Lcr : 0.0;  // Solver3D.cuh:676
    o->free_len = in->Lcr;  // Solver3D.cuh:989
    o->total_rt = in->total_rt;
    o->rt_index = 0;
    o->eom_beta = in->eom_beta;
    o->eom_fpm = in->eom_fpm;
    o->t_window = in->t_window > 0 ? in->t_window : trt;

    if (sc) {
        const double vals[OR_N_SCALARS] = {n[0], n[1], n[2], v[0], v[1], v[2], b2[0], b2[1], b2[2],
                                           b3[0], b3[1], b3[2], dQ, dk, dx, dy, dz, kp, ks, ki,
                                           kappa[0], kappa[1], kappa[2], trt, dt, (double)nsteps};
        std::memcpy(sc, vals, sizeof(vals));
    }

    const double T = in->t_window > 0 ? in->t_window : trt;
    std::vector<double> tt(nt), F(nt), ww(nt);
    for (int i = 0; i < nt; i++) tt[i] = -T * 0.5 + i * (T * 0.5 - (-T * 0.5)) / (nt - 1);
    const double fmin = -0.5 * nt / T, fmax = +0.5 * nt / T;
    for (int i = 0; i < nt; i++) F[i] = fmin + i * (fmax - fmin) / (nt - 1);
    const int c = nt / 2;
    for (int i = 0; i < nt / 2; i++) { ww[i + c] = F[i]; ww[i] = F[i + c]; }
    for (int i = 0; i < nt; i++) ww[i] *= (2.0 * PI);
    if (t) std::memcpy(t, tt.data(), sizeof(double) * nt);
    if (w) std::memcpy(w, ww.data(), sizeof(double) * nt);

    if (Api) {
        const double P = in->P, w0 = in->w0;
        const double tau = in->FWHM * std::sqrt(2.0) / (2 * std::sqrt(2 * std::log(2.0)));
        const double w02 = w0 * w0;
        const double zR = PI * n[0] * w02 / lp;
        const double eta = in->focal / zR;
        // 1-D (nx = ny = 1): EFields1D.cuh:145-148, mean intensity 2P/(pi w0^2), no focusing
        const bool one_d = nx == 1 && ny == 1;
        if (one_d && (in->pump_mode == OR_PUMP_FOCUSED_CW || in->pump_mode == OR_PUMP_FOCUSED_PULSED ||
                      in->pump_mode == OR_PUMP_FOCUSED_SECH2))
            return -3;
        const double pk = one_d ? 2.0 : 4.0;
        const double Ap0 = std::sqrt(pk * P / (EPS0 * C * PI * n[0] * w02));
        const cd MX(1, -eta);
        const double uX = 0.5 * nx, uY = 0.5 * ny;
        // sech^2 envelopes: |A|^2 ~ sech^2(t/ts), FWHM = 2 acosh(sqrt 2) ts; P is then the
        // window-average power, so the peak is P T / (2 ts).
        const double ts = in->FWHM / (2 * std::acosh(std::sqrt(2.0)));
        const double Ap0s = std::sqrt(pk * (P * T / (2 * ts)) / (EPS0 * C * PI * n[0] * w02));
        for (int it = 0; it < nt; it++)
            for (int y = 0; y < ny; y++)
                for (int x = 0; x < nx; x++) {
                    double rx = (x - uX) * dx, ry = (y - uY) * dy;
                    double r2 = rx * rx + ry * ry;
                    double tn = tt[it] / tau;
                    cd val;
                    switch (in->pump_mode) {
                    case OR_PUMP_WAVEPLANE_CW:  // EFields3D.cuh:72-85
                        val = cd(Ap0 * std::exp((-rx * rx - ry * ry) / (w0 * w0)), 0);
                        break;
                    case OR_PUMP_WAVEPLANE_PULSED:  // EFields3D.cuh:89-103
                        val = cd(Ap0 * std::exp(-tn * tn - r2 / (w0 * w0)), 0);
                        break;
                    case OR_PUMP_FOCUSED_CW:  // EFields3D.cuh:107-120
                        val = realDiv(Ap0, MX) * cpxExp(realDiv(-rx * rx - ry * ry, w02 * MX));
                        break;
                    case OR_PUMP_FOCUSED_PULSED:  // EFields3D.cuh:124-137
                        val = realDiv(Ap0, MX) * std::exp(-tn * tn) *
                              cpxExp(realDiv(-rx * rx - ry * ry, w02 * MX));
                        break;
                    case OR_PUMP_FOCUSED_SECH2:
                        val = realDiv(Ap0s, MX) / std::cosh(tt[it] / ts) *
                              cpxExp(realDiv(-rx * rx - ry * ry, w02 * MX));
                        break;
                    case OR_PUMP_WAVEPLANE_SECH2:
                        val = cd(Ap0s / std::cosh(tt[it] / ts) * std::exp(-r2 / w02), 0);
                        break;
                    default:
                        return -3;
                    }
                    size_t id = (size_t)it * nx * ny + (size_t)y * nx + x;
                    Api[2 * id] = val.real();
                    Api[2 * id + 1] = val.imag();
                }
    }
    return 0;
}

// Single pass, Solver3D.cuh:1031-1043 (propagators set as :550-567 and :700-721).
int or_single_pass(const OrParams *p, const double *w, double *Ap, double *As, double *Ai)
{
    Run r(p, w);
    cd *F[3] = {reinterpret_cast<cd *>(Ap), reinterpret_cast<cd *>(As), reinterpret_cast<cd *>(Ai)};
    r.ssfm(F);
    return 0;
}

// Round trips, Solver3D.cuh:979-1011:
//   Ap <- Api; SSFM; if not the last round trip: free-space return of s and i by +Lcr
//   (scale 1/(NX NY)); EOM on s and i, exp(i beta sin(2 pi fpm t)) (the 1-D solver's
//   intracavity modulator, Solver1D.cuh:63-72,467; it acts per t-plane, so it commutes
//   with the free-space return); GDD on s and i (fixed form of :644-694); mirrors
//   sqrt(R) e^{i phase} on the resonant s and i (Cavity3D.cuh:12-28,68-80).
int or_round_trips(OrParams *p, const double *w, const double *Api, double *Ap, double *As,
                   double *Ai, int n_rt)
{
    Run r(p, w);
    const size_t V = (size_t)p->nx * p->ny * p->nt;
    cd *F[3] = {reinterpret_cast<cd *>(Ap), reinterpret_cast<cd *>(As), reinterpret_cast<cd *>(Ai)};
    for (int k = 0; k < n_rt; k++) {
        std::memcpy(Ap, Api, sizeof(double) * 2 * V);
        r.ssfm(F);
        if (p->rt_index != p->total_rt - 1 && (p->flags & OR_DIFFRACTION))
            xyOp(p, r.cache, F, r.freeTab, 6u, 1.0 / ((double)p->nx * p->ny));
        if (p->eom_beta != 0) {
            const size_t plane = (size_t)p->nx * p->ny;
            const double T = p->t_window;
            for (int it = 0; it < p->nt; it++) {
                const double t = -T * 0.5 + it * (T * 0.5 - (-T * 0.5)) / (p->nt - 1);
                const cd e = cpxExp(p->eom_beta * std::sin(2 * PI * p->eom_fpm * t));
                for (size_t v = (size_t)it * plane; v < (size_t)(it + 1) * plane; v++) {
                    F[1][v] *= e;
                    F[2][v] *= e;
                }
            }
        }
        if (p->gdd != 0 && (p->flags & OR_DISPERSION)) {
            OrParams q = *p;
            q.flags &= ~(unsigned)OR_ASIS_Q2;
            tAxisOp(&q, r.cache, F, r.gddTab, 6u);
        }
        // only resonant fields meet a mirror (Solver3D.cuh:993-994)
        const cd ms = (p->resonant & 2u) ? std::sqrt(p->Rs) * cpxExp(p->detuning) : cd(1, 0);
        const cd mi = (p->resonant & 4u) ? std::sqrt(p->Ri) * cpxExp(p->detuning) : cd(1, 0);
#pragma omp parallel for schedule(static)
        for (long long v = 0; v < (long long)V; v++) {
            F[1][v] = ms * F[1][v];
            F[2][v] = mi * F[2][v];
        }
        p->rt_index++;
    }
    return 0;
}

}  // extern "C"
