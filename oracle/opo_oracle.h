/* Test infrastructure, NOT product code.
 *
 * FP64 CPU oracle for the cuOPO3D split-step Fourier solver (three coupled chi(2)
 * fields).  It restates the reference algorithm step by step (each function cites
 * the reference file:line it follows, paths relative to alfredos84/cuOPO3D) and is
 * used only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, as
 * the checker.  The product never links or calls it.
 *
 * Parity status: pinned against outputs of the reference itself (its own headers
 * compiled by oracle/refharness, run on a B200) through the fixtures in tests/golden.
 *
 * Fields are interleaved complex128 (re, im) arrays in the reference layout
 * [t][y][x], x fastest (reference Common.cuh:167-170).
 */
#ifndef OPO_ORACLE_H
#define OPO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Semantics flags. */
enum {
    OR_DISPERSION = 1u << 0, /* t-axis linear step (reference -DDISPERSION)           */
    OR_DIFFRACTION = 1u << 1, /* (x,y) linear step (reference -DDIFFRACTION)          */
    OR_PHYSICS = 1u << 2,    /* fixed physics: RK4 stage offsets with h, exp(i dk z),
                                absorption applied once, kp/ki from their own indices */
    OR_ASIS_Q1 = 1u << 3,    /* diffraction inverse scale 1/(NX NY NT) as shipped      */
    OR_ASIS_Q2 = 1u << 4,    /* dispersion only on row y=0, scale 1/(NX NY NT)         */
    OR_TOD = 1u << 5,        /* not in the reference: w^3 b3 / 6 in the dispersion phase */
};

enum { OR_PPLN = 0, OR_MGOSPPLT = 1, OR_MGOPPLN = 2, OR_ZGP = 3 };

enum {
    OR_PUMP_WAVEPLANE_CW = 0,
    OR_PUMP_WAVEPLANE_PULSED = 1,
    OR_PUMP_FOCUSED_CW = 2,
    OR_PUMP_FOCUSED_PULSED = 3,
    OR_PUMP_FOCUSED_SECH2 = 4,   /* not in the reference: sech^2 intensity envelope */
    OR_PUMP_WAVEPLANE_SECH2 = 5, /* not in the reference */
};

/* Physical description of one run (the reference's main() parameters). */
typedef struct {
    int crystal;                 /* OR_PPLN / OR_MGOSPPLT / OR_MGOPPLN / OR_ZGP     */
    double LX, LY, Lcr, T, Lambda, lp, ls; /* um, um, um, degC, um, um, um         */
    int nx, ny, nt, nz;          /* grid, nz = slices (dz = Lcr/(nz-1)); nx = ny = 1
                                    (no diffraction) is the plane-wave 1-D solver     */
    double dQ;                   /* um/V; <= 0 keeps the crystal's 2 d33 / pi       */
    double alpha[3];             /* 1/um; < 0 keeps the crystal's value             */
    double Lcav, Rs, Ri;         /* um; mirror reflectivities                       */
    double gdd_gamma;            /* 0: no GDD compensation                          */
    double detuning;             /* mirror phase (rad)                              */
    double P, FWHM, w0, focal;   /* W (peak), ps, um, um                            */
    int pump_mode;               /* OR_PUMP_*                                       */
    double t_window;             /* ps; <= 0 uses the round-trip time               */
    unsigned flags;              /* OR_* semantics                                  */
    int zloop_f32;               /* step count from the FP32 (1) or FP64 (0) loop   */
    int n_steps;                 /* > 0 overrides the loop count (physics mode)     */
    int total_rt;                /* round trips of the run (last one skips free space) */
    unsigned pol;                /* ZGP: bit f set = wave f (p, s, i) extraordinary   */
    double eom_beta, eom_fpm;    /* intracavity EOM (Cavity1D.cuh:75-84); beta 0: none */
    unsigned resonant;           /* mirrors act on fields with bit f set (2 s, 4 i)  */
} OrPhys;

/* Everything the split-step needs, derived from OrPhys. */
typedef struct {
    int nx, ny, nt, n_steps;
    unsigned flags;
    double dz, Lcr, dx, dy;
    double kappa[3];    /* coupling p, s, i                      */
    double kdiff[3];    /* wavevectors used by diffraction       */
    double vinv[3];     /* group delay per um relative to frame  */
    double beta2[3];
    double alpha[3];
    double dk;
    double Rs, Ri, detuning, gdd, free_len;
    int total_rt;
    int rt_index;       /* round trips done so far (in/out)      */
    double beta3[3];    /* third-order dispersion (OR_TOD)       */
    double eom_beta, eom_fpm, t_window;
    unsigned resonant;
} OrParams;

/* Derived scalars, in this order (the harness dump uses the same names):
 * np ns ni vp vs vi b2p b2s b2i b3p b3s b3i dQ dk dx dy dz kp ks ki
 * kappa_p kappa_s kappa_i trt dt nsteps  (26 values) */
#define OR_N_SCALARS 26

int or_setup(const OrPhys *in, OrParams *out, double *scalars, double *t, double *w,
             double *Api);
int or_zloop_steps(double Lcr, double dz, int f32);
/* n, group velocity, GVD, TOD as the reference prints it, and the exact TOD (third
 * derivative by central difference) of one crystal index (extraordinary selects ZGP's
 * 'e'; ZGP has no reference TOD, both are the exact one). */
int or_crystal_dispersion(int crystal, double T, int extraordinary, double L, double out[5]);
void or_fft(int n, int sign, double *data);
void or_noise(uint64_t seed, double sigma, size_t n_complex, double *out);
int or_single_pass(const OrParams *p, const double *w, double *Ap, double *As, double *Ai);
int or_round_trips(OrParams *p, const double *w, const double *Api, double *Ap, double *As,
                   double *Ai, int n_rt);
void or_power_sums(int n, const double *A, double *sum_abs2);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
