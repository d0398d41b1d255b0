// Crystal classes with cuOPO3D's constructor arguments and public members.  The
// Sellmeier-derived values (index, group velocity, GVD, TOD at the three wavelengths)
// come from the library in FP64 (opo_crystal_dispersion); dx, dy, dz follow the
// compile-time grid, and kp / ki keep the shipped definitions (2 pi ns / lp, 2 pi ni / ls).
#pragma once

#include "Common.cuh"
#include "cuopo3d.h"

template <int KIND> class OpoCrystal {
public:
    static constexpr int kind = KIND;
    real_t Lcr, LX, LY, T, Lambda, lp, ls, li;
    real_t d33, dQ, alpha_crp, alpha_crs, alpha_cri, beta_crs = 0, chi3p = 0, chi3s = 0, chi3i = 0;
    real_t np, ns, ni, vp, vs, vi, b2p, b2s, b2i, b3p, b3s, b3i;
    real_t dx = 0, dy = 0, dz, kp, ks, ki, dk;
    std::string name;
    bool QPM = true;
    unsigned pol_bits = 7;  // bit f: wave f extraordinary (only ZGP has a choice)

    OpoCrystal(const char *nm, real_t d33_, real_t ap, real_t as, real_t ai, real_t _LX, real_t _LY, real_t _Lcr,
               real_t _T, real_t _Lambda, real_t _lp, real_t _ls, real_t _li, bool qpm = true,
               unsigned pol = 7)
        : Lcr(_Lcr), LX(_LX), LY(_LY), T(_T), Lambda(_Lambda), lp(_lp), ls(_ls), li(_li), d33(d33_),
          alpha_crp(ap), alpha_crs(as), alpha_cri(ai), name(nm), QPM(qpm), pol_bits(pol)
    {
        printLineOnScreen();
        std::cout << "\nInstance of the class " << name << ".\n";
        dQ = 2.0 * d33 / PI;
        dx = (real_t)(LX / (NX - 1.0f));
        dy = (real_t)(LY / (NY - 1.0f));
        dz = (real_t)(Lcr / (NZ - 1.0f));
        double o[4];
        real_t *dst[3][4] = {{&np, &vp, &b2p, &b3p}, {&ns, &vs, &b2s, &b3s}, {&ni, &vi, &b2i, &b3i}};
        const real_t lam[3] = {lp, ls, li};
        for (int f = 0; f < 3; f++) {
            if (opo_crystal_dispersion_pol(KIND, T, (pol_bits >> f) & 1u, lam[f], o) != OPO_OK) {
                std::cerr << "crystal dispersion failed" << std::endl;
                exit(1);
            }
            for (int k = 0; k < 4; k++) *dst[f][k] = (real_t)o[k];
        }
        kp = 2.0f * PI * ns / lp;
        ks = 2.0f * PI * ns / ls;
        ki = 2.0f * PI * ni / ls;
        dk = kp - ks - ki - (QPM ? 2.0f * PI / Lambda : 0.0f);
    }
    real_t n(real_t L, real_t Tc) const { return prop(L, Tc, 0); }
    real_t GV(real_t L, real_t Tc) const { return prop(L, Tc, 1); }
    real_t GVD(real_t L, real_t Tc) const { return prop(L, Tc, 2); }
    real_t TOD(real_t L, real_t Tc) const { return prop(L, Tc, 3); }
    void getCrystalProp() const
    {
        std::cout << "Crystal name = " << name << "\n        ---> Temp            = " << T << " C"
                  << "\n        ---> np, ns, ni      = " << np << ", " << ns << ", " << ni
                  << "\n        ---> vgp, vgs, vgi   = " << vp << ", " << vs << ", " << vi << " um/ps"
                  << "\n        ---> b2p, b2s, b2i   = " << b2p << ", " << b2s << ", " << b2i << " ps^2/um"
                  << "\n        ---> dQ              = " << dQ * 1e6 << " pm/V"
                  << "\n        ---> dx, dy, dz      = " << dx << ", " << dy << ", " << dz << " um"
                  << "\n        ---> Crystal length  = " << Lcr * 1e-3 << " mm\n" << std::endl;
    }

private:
    real_t prop(real_t L, real_t Tc, int k) const
    {
        double o[4] = {0, 0, 0, 0};
        opo_crystal_dispersion(KIND, Tc, L, o);
        return (real_t)o[k];
    }
};

// Congruent PPLN (Jundt Sellmeier), cuOPO3D CrystalsBase/PPLN.cuh.
class PPLN : public OpoCrystal<OPO_PPLN> {
public:
    PPLN(real_t LX, real_t LY, real_t Lcr, real_t T, real_t Lambda, real_t lp, real_t ls, real_t li)
        : OpoCrystal("PPLN", 25.20e-6, 0.025e-4, 0.002e-4, 0.002e-4, LX, LY, Lcr, T, Lambda, lp, ls, li) {}
};

// MgO:sPPLT (Bruner Sellmeier), cuOPO3D CrystalsBase/MgOsPPLT.cuh.
class MgOsPPLT : public OpoCrystal<OPO_MGOSPPLT> {
public:
    MgOsPPLT(real_t LX, real_t LY, real_t Lcr, real_t T, real_t Lambda, real_t lp, real_t ls, real_t li)
        : OpoCrystal("MgOsPPLT", 11.0e-6, 1.57e-4, 0.17e-6, 0.17e-6, LX, LY, Lcr, T, Lambda, lp, ls, li) {}
};

// MgO:PPLN (Gayer Sellmeier), cuOPO3D CrystalsBase/MgOPPLN.cuh.
class MgOPPLN : public OpoCrystal<OPO_MGOPPLN> {
public:
    MgOPPLN(real_t LX, real_t LY, real_t Lcr, real_t T, real_t Lambda, real_t lp, real_t ls, real_t li)
        : OpoCrystal("MgO:PPLN", 25.20e-6, 0.025e-4, 0.002e-4, 0.002e-4, LX, LY, Lcr, T, Lambda, lp, ls, li) {}
};

// ZnGeP2 (Zelmon Sellmeier), cuOPO3D CrystalsBase/ZGP.cuh: birefringent phase matching
// with a polarisation tuple such as ('e','e','o'); no temperature, no grating.
class ZGP : public OpoCrystal<OPO_ZGP> {
public:
    std::tuple<char, char, char> pol;
    ZGP(real_t LX, real_t LY, real_t Lcr, std::tuple<char, char, char> _pol, real_t lp, real_t ls, real_t li)
        : OpoCrystal("ZPG", 75.0e-6, 1.57e-4, 0.17e-6, 0.17e-6, LX, LY, Lcr, 0, 1, lp, ls, li, false, bits(_pol)),
          pol(_pol) {}
    // ZGP.cuh:98-102: stores the tuple; the indices keep their constructed values
    void setPolarizations(char p, char s, char i) { pol = std::make_tuple(p, s, i); }
    real_t n(real_t L, char pc) const { return prop(L, pc, 0); }
    real_t GV(real_t L, char pc) const { return prop(L, pc, 1); }
    real_t GVD(real_t L, char pc) const { return prop(L, pc, 2); }

private:
    static unsigned bits(const std::tuple<char, char, char> &p)
    {
        return (std::get<0>(p) == 'e' ? 1u : 0u) | (std::get<1>(p) == 'e' ? 2u : 0u) |
               (std::get<2>(p) == 'e' ? 4u : 0u);
    }
    real_t prop(real_t L, char pc, int k) const
    {
        double o[4] = {0, 0, 0, 0};
        opo_crystal_dispersion_pol(OPO_ZGP, 0, pc == 'e', L, o);
        return (real_t)o[k];
    }
};
