// Ring cavity with cuOPO3D's constructor and members (round-trip time, GDD flag, mirror).
#pragma once

#include "EFields3D.cuh"

struct OpoMirror {
    float2 m;
    __host__ __device__ cuFloatComplex operator()(const cuFloatComplex &a) const
    {
        return make_cuFloatComplex(m.x * a.x - m.y * a.y, m.x * a.y + m.y * a.x);
    }
};

template <typename Crystal> class Cavity {
public:
    real_t Rs, Ri, Lcav, Lfs, trt, fsr, dt;
    real_t gamma = 0;
    real_t beta = 0, fpm = 0;
    bool gdd = false, satabs = false, eom = false;
    real_t detuning = 0;  // round-trip phase at the mirrors (0 in cuOPO3D)
    Crystal *Cr;

    Cavity(Crystal *_Cr, real_t _Lcav, real_t _Rs, real_t _Ri) : Rs(_Rs), Ri(_Ri), Lcav(_Lcav), Cr(_Cr)
    {
        trt = (Lcav + (Cr->Lcr) * ((Cr->ns) - 1)) / C;
        dt = trt / (NT - 1);
        fsr = 1. / trt;
        Lfs = Lcav - Cr->Lcr;
        printLineOnScreen();
        std::cout << "\nInstance of the class Cavity." << std::endl;
    }
    ~Cavity() {}

    // A <- sqrt(R) e^{i phase} A on the device.
    void applyReflectivity(cVecd_t &A, real_t R, real_t phase)
    {
        OpoMirror f{make_float2(std::sqrt(R) * std::cos(phase), std::sqrt(R) * std::sin(phase))};
        thrust::transform(A.begin(), A.end(), A.begin(), f);
        opo_files::invalidate();
    }
    void setGDDCompensation(real_t g)
    {
        gdd = true;
        gamma = g;
    }
    // Intracavity electro-optic modulator (cuOPO3D Cavity1D.cuh:75-84): after the crystal,
    // signal and idler x exp(i beta sin(2 pi fpm t)), before GDD and the mirrors.
    void setEOM(real_t _beta, real_t _fpm)
    {
        eom = true;
        beta = _beta;
        fpm = _fpm;
        std::cout << "Set intracavity EOM:\n        ---> beta = " << beta << "\n        ---> fpm = " << fpm * 1e3
                  << " GHz" << std::endl;
    }
    void getCavityProp() const
    {
        std::cout << "Set OPO cavity:\n        ---> Cavity length         = " << Lcav * 1e-6 << " m"
                  << "\n        ---> Round trip time       = " << trt << " ps"
                  << "\n        ---> Free spectral range   = " << fsr * 1e3 << " GHz"
                  << "\n        ---> Signal reflectivity   = " << Rs * 100 << " %"
                  << "\n        ---> Idler reflectivity    = " << Ri * 100 << " %" << std::endl;
        if (gdd) std::cout << "        ---> Set " << (int)(100 * gamma) << "% Intracavity GDD compensation." << std::endl;
    }
};
