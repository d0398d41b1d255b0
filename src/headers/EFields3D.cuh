// EFields with cuOPO3D's constructor and members.  Api / Ap / As / Ai stay Thrust device
// vectors of complex_t in the [t][y][x] layout, so existing savers and host code work;
// the pump and the grids are computed in FP64 by the library.
#pragma once

#include "Crystals.cuh"

template <typename Crystal> class EFields {
public:
    cVecd_t Api, Ap, As, Ai;
    rVecd_t t, F, w;
    real_t lp, ls, li, waist, Power;
    real_t np, ns, ni, vp, vs, vi, b2p, b2s, b2i;
    real_t alpha_crp, alpha_crs, alpha_cri;
    real_t kp, ks, ki, kappa_p, kappa_s, kappa_i;
    real_t dx, dy, dz, dk, dkp;
    std::tuple<bool, bool, bool> resFields{false, true, true};
    Crystal *Cr;
    // recorded for the solver
    double window = 0;
    OpoConfig pump_cfg{};
    bool pump_set = false;

    EFields(real_t _lp, real_t _ls, real_t _li, real_t _Power, real_t _waist, Crystal *_Cr)
        : lp(_lp), ls(_ls), li(_li), waist(_waist), Power(_Power), Cr(_Cr)
    {
        Api.resize(SIZE); Ap.resize(SIZE); As.resize(SIZE); Ai.resize(SIZE);
        t.resize(NT); F.resize(NT); w.resize(NT);
        printLineOnScreen();
        std::cout << "\nInstance of the class Efields." << std::endl;
        np = Cr->np; ns = Cr->ns; ni = Cr->ni;
        vp = Cr->vp; vs = Cr->vs; vi = Cr->vi;
        b2p = Cr->b2p; b2s = Cr->b2s; b2i = Cr->b2i;
        alpha_crp = Cr->alpha_crp; alpha_crs = Cr->alpha_crs; alpha_cri = Cr->alpha_cri;
        dx = Cr->dx; dy = Cr->dy; dz = Cr->dz;
        kappa_p = 2 * PI * Cr->dQ / (np * lp);
        kappa_s = 2 * PI * Cr->dQ / (ns * ls);
        kappa_i = 2 * PI * Cr->dQ / (ni * li);
        kp = 2.0f * PI * ns / lp;
        ks = 2.0f * PI * ns / ls;
        ki = 2.0f * PI * ni / ls;
        dk = Cr->dk;
        dkp = 1 / vp - 1 / vs;
    }
    ~EFields() {}

    // The configuration of this field set (grid, crystal, window, pump) for the library.
    OpoConfig config() const
    {
        OpoConfig c = pump_set ? pump_cfg : OpoConfig{};
        c.crystal = Crystal::kind;
        c.pol = Cr->pol_bits;
        c.LX = Cr->LX; c.LY = Cr->LY; c.Lcr = Cr->Lcr; c.T = Cr->T; c.Lambda = Cr->Lambda;
        c.lp = lp; c.ls = ls;
        c.nx = NX; c.ny = NY; c.nt = NT; c.nz = NZ;
        c.dQ = Cr->dQ;
        c.alpha[0] = Cr->alpha_crp; c.alpha[1] = Cr->alpha_crs; c.alpha[2] = Cr->alpha_cri;
        c.t_window = window;
        return c;
    }

    void setTimeFreqVectors(real_t trt)
    {
        std::cout << "\t---> Setting time and frequency vectors...";
        window = trt;
        std::vector<double> tt(NT), ww(NT);
        opo_time_freq(NT, trt, tt.data(), ww.data());
        rVech_t th(tt.begin(), tt.end()), wh(ww.begin(), ww.end()), fh(NT);
        for (uint32_t i = 0; i < NT; i++) fh[i] = (real_t)(-0.5 * NT / trt + i * (NT / trt) / (NT - 1));
        t = th; w = wh; F = fh;
        std::cout << "done.\n" << std::flush;
    }

    void setPumpField(real_t P, real_t FWHM, real_t w0, real_t focal, std::string mode)
    {
        static const char *names[] = {"waveplane-cw", "waveplane-pulsed", "focused-cw", "focused-pulsed",
                                      "focused-sech2", "waveplane-sech2"};
        int m = -1;
        for (int k = 0; k < 6; k++)
            if (mode == names[k]) m = k;
        if (m < 0) {
            std::cout << "Invalid option for pump electric field!!\n";
            return;
        }
        pump_cfg = config();
        pump_cfg.P = P; pump_cfg.FWHM = FWHM; pump_cfg.w0 = w0; pump_cfg.focal = focal; pump_cfg.pump_mode = m;
        pump_cfg.Lcav = -1; pump_cfg.precision = OPO_FP32; pump_cfg.flags = OPO_DISPERSION | OPO_DIFFRACTION;
        std::vector<double> a(2 * (size_t)SIZE);
        if (opo_pump_field(&pump_cfg, a.data()) != OPO_OK) {
            std::cerr << "pump field: invalid configuration" << std::endl;
            exit(1);
        }
        cVech_t h(SIZE);
        for (size_t k = 0; k < SIZE; k++) h[k] = make_cuFloatComplex((float)a[2 * k], (float)a[2 * k + 1]);
        Api = h;
        pump_set = true;
        opo_files::invalidate();
        std::cout << "        ---> Pump field mode: " << mode << "\n        ---> Pump Power: " << P
                  << " W\n        ---> Beam waist: " << w0 << " um\n" << std::endl;
    }
    void setPumpField(real_t P, real_t FWHM, real_t w0, std::string mode) { setPumpField(P, FWHM, w0, Cr->Lcr / 2, mode); }

    // Seeded noise N(0, 1e-15) per component (the reference seeds from the wall clock);
    // the seed can be set with the environment variable OPO_NOISE_SEED.
    void noiseGenerator(cVecd_t &Vec)
    {
        const char *env = std::getenv("OPO_NOISE_SEED");
        const uint64_t seed = env ? std::strtoull(env, nullptr, 10) : 1;
        std::vector<double> a(2 * Vec.size());
        opo_noise(seed, 1.0e-15, Vec.size(), a.data());
        cVech_t h(Vec.size());
        for (size_t k = 0; k < h.size(); k++) h[k] = make_cuFloatComplex((float)a[2 * k], (float)a[2 * k + 1]);
        Vec = h;
        opo_files::invalidate();
    }
};
