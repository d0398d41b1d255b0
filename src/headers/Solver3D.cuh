// Solver with cuOPO3D's constructors and methods.  runOPO / runSinglePass hand the
// EFields device vectors to the cuopo3d-b200 library (device-to-device, no host copy),
// run the split-step there and copy the results back into the same vectors.  The bulk
// fields run in FP32 like the shipped build; compile with -DOPO_DROPIN_FP64 for the FP64
// form (the device vectors stay complex64).
#pragma once

#include <thrust/transform_reduce.h>

#include "Cavity3D.cuh"

struct OpoAbs2 {
    __host__ __device__ double operator()(const cuFloatComplex &a) const
    {
        return (double)a.x * a.x + (double)a.y * a.y;
    }
};

template <typename Crystal> class Solver {
public:
    Crystal *Cr;
    EFields<Crystal> *A;
    Cavity<Crystal> *Cav = nullptr;

    Solver(Crystal *_Cr, EFields<Crystal> *_A) : Cr(_Cr), A(_A) { banner(false); }
    Solver(Crystal *_Cr, Cavity<Crystal> *_Cav, EFields<Crystal> *_A) : Cr(_Cr), A(_A), Cav(_Cav) { banner(true); }
    ~Solver() {}

    bool checkCourantStability(real_t dz, real_t kpdxdy) const { return dz < kpdxdy; }

    real_t averagePowerCutXY(const cVecd_t &F) const
    {
        const double s = thrust::transform_reduce(F.begin(), F.end(), OpoAbs2(), 0.0, thrust::plus<double>());
        return (real_t)(0.5 * EPS0 * C * Cr->ns * Cr->dx * Cr->dy / (Cr->LX * Cr->LY) * s);
    }

    void runOPO(const std::vector<int> &) { runOPO(); }
    void runOPO()
    {
        if (!checkCourantStability(Cr->dz, 0.2f * A->kp * Cr->dx * Cr->dy)) {
            std::cout << "        ---> Courant convergence criteria: failed.\n        ---> Please change step sizes."
                      << std::endl;
            return;
        }
        std::cout << "        ---> Courant convergence criteria: passed" << std::endl;
        run(true);
    }
    void runSinglePass() { run(false); }

private:
    void banner(bool cavity) const
    {
        printLineOnScreen();
        std::cout << "\nInstance of the class Solver.\n";
        if (cavity) std::cout << "        ---> Number of roundtrips: " << NRT << "\n";
        std::cout << "        ---> Number of crystal slices: " << NZ << std::endl;
    }

    static void check(int rc, OpoSolver *s, const char *what)
    {
        if (rc != OPO_OK) {
            std::cerr << what << ": " << opo_last_error(s) << std::endl;
            exit(1);
        }
    }

    void run(bool opo)
    {
        OpoConfig c = A->config();
        unsigned flags = 0;
#ifdef DISPERSION
        flags |= OPO_DISPERSION;
#endif
#ifdef DIFFRACTION
        flags |= OPO_DIFFRACTION;
#endif
        c.flags = flags;
        c.zloop_f32 = 1;  // step count of the shipped FP32 z loop
        c.total_rt = opo ? NRT : 1;
#ifdef OPO_DROPIN_FP64
        c.precision = OPO_FP64;
#else
        c.precision = OPO_FP32;
#endif
        c.resonant = (std::get<1>(A->resFields) ? 2u : 0u) | (std::get<2>(A->resFields) ? 4u : 0u);
        if (Cav) {
            c.Lcav = Cav->Lcav; c.Rs = Cav->Rs; c.Ri = Cav->Ri;
            c.gdd_gamma = Cav->gdd ? Cav->gamma : 0.0;
            c.detuning = Cav->detuning;
            c.eom_beta = Cav->eom ? Cav->beta : 0.0;
            c.eom_fpm = Cav->eom ? Cav->fpm : 0.0;
        } else {
            c.Lcav = -1; c.Rs = 1; c.Ri = 1; c.resonant = 0;
        }
        OpoParams p;
        check(opo_params_from_config(&c, &p, nullptr), nullptr, "configuration");
        std::vector<double> w(NT);
        opo_time_freq(NT, p.t_window, nullptr, w.data());
        OpoSolver *s = nullptr;
        check(opo_create(&p, w.data(), &s), nullptr, "solver");
        check(opo_autotune(s), s, "autotune");
        const int which[4] = {OPO_FIELD_PUMP_INITIAL, OPO_FIELD_PUMP, OPO_FIELD_SIGNAL, OPO_FIELD_IDLER};
        cVecd_t *vec[4] = {&A->Api, &A->Ap, &A->As, &A->Ai};
        for (int k = 0; k < 4; k++)
            check(opo_set_field(s, which[k], thrust::raw_pointer_cast(vec[k]->data()), OPO_MEM_DEVICE, OPO_FP32), s,
                  "upload");
        const double t0 = seconds();
        check(opo ? opo_run_round_trips(s, NRT) : opo_run_single_pass(s), s, "run");
        check(opo_synchronize(s), s, "run");
        double sums[3];
        const int frc = opo_field_sums(s, sums);
        if (frc == OPO_ERR_NONFINITE)
            std::cout << "Simulation failed. Error in NaN check after the last round trip." << std::endl;
        for (int k = 1; k < 4; k++)
            check(opo_get_field(s, which[k], thrust::raw_pointer_cast(vec[k]->data()), OPO_MEM_DEVICE, OPO_FP32), s,
                  "download");
        check(opo_synchronize(s), s, "download");
        opo_files::invalidate();
        TimingCode(seconds() - t0);
        opo_destroy(s);
    }
};
