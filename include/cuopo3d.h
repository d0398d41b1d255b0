/* cuopo3d.h -- C-ABI of the B200-native split-step Fourier solver for three coupled
 * chi(2) fields (pump, signal, idler) in an optical parametric oscillator.
 *
 * This is the boundary a caller binds (C, C++, ctypes, cgo ...): plain pointers,
 * sizes and int status codes; no CUDA or torch types.  It replaces the C++ template
 * interface of alfredos84/cuOPO3D (src/headers), whose classes keep working through
 * the drop-in headers in src/headers of this repository.  Each entry point names the
 * reference interface it stands in for (file:line, paths in that project).
 *
 * Layout: every field is a complex array in the reference order [t][y][x], x fastest
 * (reference src/headers/Common.cuh:167-170).  Host-side complex values are
 * interleaved (re, im) doubles (OPO_FP64) or floats (OPO_FP32).
 *
 * Threading: one host thread per solver; solvers are independent; calls on one
 * solver are ordered on its CUDA stream.  Errors never exit the process: every call
 * returns an OPO_* status and opo_last_error() explains the last failure.
 */
#ifndef CUOPO3D_H
#define CUOPO3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------ */
enum {
    OPO_OK = 0,
    OPO_ERR_INVALID = 1,     /* bad argument or unsupported size                      */
    OPO_ERR_CUDA = 2,        /* a CUDA runtime call failed                            */
    OPO_ERR_NOMEM = 3,       /* device allocation failed                              */
    OPO_ERR_NONFINITE = 4,   /* a field became NaN/Inf (reference Solver3D.cuh:999-1005) */
    OPO_ERR_COURANT = 5,     /* reference step-size gate failed (Solver3D.cuh:973,1016-1019) */
    OPO_ERR_CAPACITY = 6     /* request exceeds a fixed capacity                      */
};

/* ---- semantics flags (OpoConfig.flags / OpoParams.flags) ----------------------- */
enum {
    OPO_DISPERSION = 1u << 0,  /* t-axis step: reference -DDISPERSION (cuOPO3D.sh:38)   */
    OPO_DIFFRACTION = 1u << 1, /* (x,y) step: reference -DDIFFRACTION (cuOPO3D.sh:38)   */
    OPO_PHYSICS = 1u << 2,     /* corrected physics: RK4 stages with h, exp(i dk z),
                                  absorption once, kp/ki from their own indices       */
    OPO_ASIS_Q1 = 1u << 3,     /* shipped diffraction scale 1/(NX NY NT)
                                  (Solver3D.cuh:83,780)                                 */
    OPO_ASIS_Q2 = 1u << 4,     /* shipped dispersion on row y=0 only, scale 1/(NX NY NT)
                                  (Solver3D.cuh:603,613,616,629)                        */
    OPO_TOD = 1u << 5          /* third-order dispersion: the t-axis phase gains
                                  dz w^3 b3 / 6 (b3 of PPLN.cuh:73 etc., which the
                                  reference computes but never applies)                 */
};

enum { OPO_FP32 = 0, OPO_FP64 = 1 };                  /* bulk field precision          */
enum {                                                 /* crystal models (Crystals.cuh)  */
    OPO_PPLN = 0,      /* CrystalsBase/PPLN.cuh (Jundt)                         */
    OPO_MGOSPPLT = 1,  /* CrystalsBase/MgOsPPLT.cuh (Bruner)                    */
    OPO_MGOPPLN = 2,   /* CrystalsBase/MgOPPLN.cuh (Gayer)                      */
    OPO_ZGP = 3        /* CrystalsBase/ZGP.cuh (Zelmon; o/e per wave, no QPM)   */
};
enum {                                                 /* pump profiles                 */
    OPO_PUMP_WAVEPLANE_CW = 0,     /* EFields3D.cuh:72-85    */
    OPO_PUMP_WAVEPLANE_PULSED = 1, /* EFields3D.cuh:89-103   */
    OPO_PUMP_FOCUSED_CW = 2,       /* EFields3D.cuh:107-120  */
    OPO_PUMP_FOCUSED_PULSED = 3,   /* EFields3D.cuh:124-137  */
    OPO_PUMP_FOCUSED_SECH2 = 4,    /* new: sech^2 intensity, P = window-average power */
    OPO_PUMP_WAVEPLANE_SECH2 = 5   /* new */
};
enum {                                                 /* field selectors               */
    OPO_FIELD_PUMP_INITIAL = 0,    /* EFields::Api */
    OPO_FIELD_PUMP = 1,            /* EFields::Ap  */
    OPO_FIELD_SIGNAL = 2,          /* EFields::As  */
    OPO_FIELD_IDLER = 3            /* EFields::Ai  */
};
enum { OPO_MEM_HOST = 0, OPO_MEM_DEVICE = 1 };

/* ---- physical description (the knobs of the reference main(), cuOPO3D.cu:15-51) --- */
typedef struct OpoConfig {
    int crystal;                       /* OPO_PPLN / OPO_MGOSPPLT                         */
    double LX, LY, Lcr, T, Lambda;     /* um, um, um, degC, um                            */
    double lp, ls;                     /* pump, signal wavelength (um); li = ls lp/(ls-lp) */
    int nx, ny, nt, nz;                /* grid; nz slices, dz = Lcr/(nz-1); nx = ny = 1 without
                                          OPO_DIFFRACTION is the plane-wave 1-D solver
                                          (Solver1D.cuh), nt up to one tile per CTA;
                                          nx ny nt <= 2^31 - 1                           */
    double dQ;                         /* um/V; <= 0 keeps the crystal's 2 d33/pi          */
    double alpha[3];                   /* 1/um; < 0 keeps the crystal's value              */
    double Lcav, Rs, Ri;               /* cavity length (um); mirror reflectivities        */
    double gdd_gamma;                  /* GDD compensation fraction, 0 = off               */
    double detuning;                   /* round-trip phase at the mirrors (rad)            */
    double P, FWHM, w0, focal;         /* W, ps, um, um                                     */
    int pump_mode;                     /* OPO_PUMP_*                                        */
    double t_window;                   /* ps; <= 0: the cavity round-trip time             */
    unsigned flags;                    /* OPO_DISPERSION | OPO_DIFFRACTION | ...           */
    int zloop_f32;                     /* step count from the shipped FP32 z loop (1) or FP64 (0) */
    int n_steps;                       /* > 0: explicit z-step count (dz = Lcr/n_steps in physics mode) */
    int total_rt;                      /* round trips of the run (the last skips free space) */
    int precision;                     /* OPO_FP32 / OPO_FP64                               */
    unsigned resonant;                 /* bit1 signal, bit2 idler (reference resFields)     */
    unsigned pol;                      /* bit f: wave f (pump, signal, idler) extraordinary;
                                          ZGP only (its pol tuple, ZGP.cuh:24,49)          */
    double eom_beta, eom_fpm;          /* intracavity electro-optic modulator, Cavity::setEOM
                                          (Cavity1D.cuh:75-84): after the crystal, signal and
                                          idler x exp(i beta sin(2 pi fpm t)) before GDD and
                                          mirrors (Solver1D.cuh:63-72,467); beta 0: none;
                                          fpm in 1/ps                                       */
} OpoConfig;

/* ---- derived solver parameters (what the split-step consumes) ------------------- */
typedef struct OpoParams {
    int nx, ny, nt, n_steps;
    unsigned flags;
    int precision;
    double dz, Lcr, dx, dy;
    double kappa[3];   /* coupling, EFields3D.cuh:219-221                               */
    double kdiff[3];   /* wavevectors of the diffraction propagator, EFields3D.cuh:222-224 */
    double vinv[3];    /* group delay relative to the frame, Solver3D.cuh:163-165         */
    double beta2[3];
    double alpha[3];
    double dk;
    double Rs, Ri, detuning, gdd, free_len;
    unsigned resonant;
    int total_rt;
    double t_window;
    double beta3[3];   /* third-order dispersion (applied with OPO_TOD)                  */
    double eom_beta, eom_fpm;
} OpoParams;

/* Derived scalars written by opo_params_from_config (reference names, in order):
 * np ns ni vp vs vi b2p b2s b2i b3p b3s b3i dQ dk dx dy dz kp ks ki
 * kappa_p kappa_s kappa_i trt dt nsteps */
#define OPO_N_SCALARS 26

typedef struct OpoSolver OpoSolver;

/* ---- host physics (the reference's constructors) --------------------------------- */

/* Crystal, EFields and Cavity constructors in one: Sellmeier indices, group
 * velocities, GVD, TOD, kappa, k, dk, steps, round-trip time and the z-step count.
 * Replaces PPLN::PPLN (CrystalsBase/PPLN.cuh:51-78), MgOsPPLT::MgOsPPLT
 * (CrystalsBase/MgOsPPLT.cuh:51-78), EFields::EFields (EFields3D.cuh:199-227) and
 * Cavity::Cavity (Cavity3D.cuh:42-49).  scalars may be NULL. */
int opo_params_from_config(const OpoConfig *cfg, OpoParams *out, double *scalars);

/* Refractive index n, group velocity, GVD and TOD of a crystal at one wavelength
 * (PPLN.cuh:97-259, MgOsPPLT.cuh:96-226, MgOPPLN.cuh:97-259, ZGP.cuh:103-245; ZGP
 * defines no TOD, its b3 here is the same derivative formula on its Sellmeier form).
 * out = {n, vg, b2, b3}.  The extraordinary index (ZGP: pol 'e'). */
int opo_crystal_dispersion(int crystal, double T, double lambda_um, double out[4]);
/* The same for one polarisation (extraordinary = 0: ordinary; QPM crystals ignore it). */
int opo_crystal_dispersion_pol(int crystal, double T, int extraordinary, double lambda_um, double out[4]);

/* Time and angular-frequency grids, EFields::setTimeFreqVectors
 * (EFields3D.cuh:319-328): t = linspace(-T/2, T/2), w = 2 pi fftshift(linspace(
 * -nt/(2T), nt/(2T))).  Either pointer may be NULL. */
int opo_time_freq(int nt, double window, double *t, double *w);
/* The reference's average power of a field over an (x, y) cut, Solver::averagePowerCutXY
 * (Solver3D.cuh:527-536), from FP64 tallies sums[f] = sum |A_f|^2 (opo_field_sums,
 * opo_batch_sums): power[f] = 0.5 eps0 c ns dx dy / (LX LY) sums[f]. */
int opo_power_cut_xy(const OpoConfig *cfg, const double sums[3], double power[3]);

/* Initial pump field, EFields::setPumpField (EFields3D.cuh:244-296), into
 * Api (interleaved complex128, nx*ny*nt values). */
int opo_pump_field(const OpoConfig *cfg, double *Api);

/* Seeded noise replacing EFields::noiseGenerator (EFields3D.cuh:300-315): each
 * component is sigma (sum of 12 splitmix64 uniforms - 6); deterministic everywhere. */
int opo_noise(uint64_t seed, double sigma, size_t n_complex, double *out);

/* ---- solver ------------------------------------------------------------------------ */

/* Allocate the resident fields, phase tables and FFT plans on the current device.
 * w: nt angular frequencies (host doubles, opo_time_freq).  Replaces
 * Solver::Solver (Solver3D.cuh:456-468) plus setDispersionPropagators (:550-567)
 * and setDiffractionPropagators (:700-721), which are built once here. */
int opo_create(const OpoParams *p, const double *w, OpoSolver **out);
void opo_destroy(OpoSolver *s);

/* Copy a field in or out.  where = OPO_MEM_HOST / OPO_MEM_DEVICE; elem_precision
 * is the caller buffer's precision (converted on the device if it differs).
 * Stands in for the thrust assignments on EFields::Api/Ap/As/Ai
 * (cuOPO3D.cu:46,51; Solver3D.cuh:981). */
int opo_set_field(OpoSolver *s, int which, const void *src, int where, int elem_precision);
int opo_get_field(OpoSolver *s, int which, void *dst, int where, int elem_precision);

/* Initialise the fields on the device from the solver's configuration: Api = Ap = the
 * pump of opo_pump_field (EFields::setPumpField, EFields3D.cuh:244-296), As = the noise of
 * opo_noise(seed, sigma) (bit-identical), Ai = 0, or As when idler_copy (cuOPO3D.cu:51). */
int opo_init_fields(OpoSolver *s, const OpoConfig *cfg, uint64_t seed, double sigma, int idler_copy);

/* One pass through the crystal without cavity, Solver::runSinglePass
 * (Solver3D.cuh:1031-1043; SSFM :946-960). */
int opo_run_single_pass(OpoSolver *s);

/* n cavity round trips continuing from the solver's round-trip counter,
 * Solver::runOPO (Solver3D.cuh:964-1023): fresh pump, SSFM, free-space return
 * (skipped on round trip total_rt-1), GDD compensation, mirrors. */
int opo_run_round_trips(OpoSolver *s, int n);

/* Streamed round trips, for a host that feeds a solver one step after another (a sweep
 * point per step): the copies of the next step's inputs and of the last step's results
 * run on two copy streams while the round trips run, through device stages of the four
 * fields (allocated at first use: 8 x the field size).  All four calls return without
 * waiting; host buffers must be pinned and in the solver's precision, and must stay
 * untouched until opo_stream_wait.
 *   opo_stream_put  enqueue the upload of field `which` for the next opo_stream_run
 *                   (it lands in the field when that run starts);
 *   opo_stream_run  the uploaded fields go into place, n round trips run
 *                   (opo_run_round_trips), and the four fields are kept for download;
 *   opo_stream_get  enqueue the download of field `which` as the last opo_stream_run
 *                   left it (later runs do not overwrite it before it is copied);
 *   opo_stream_wait block until every streamed copy and round trip has completed.
 * No counterpart in the reference, whose main runs one configuration per process and
 * reads every saved field back with a blocking copy (cuOPO3D.cu:75-85). */
int opo_stream_put(OpoSolver *s, int which, const void *host, int elem_precision);
int opo_stream_run(OpoSolver *s, int n);
int opo_stream_get(OpoSolver *s, int which, void *host, int elem_precision);
int opo_stream_wait(OpoSolver *s);

/* FP64 sum of |A|^2 over every voxel of the pump, signal and idler (in that order);
 * the reference's averagePowerCutXY (Solver3D.cuh:529-545) is
 * 0.5 eps0 c ns dx dy / (LX LY) times the signal entry. */
int opo_field_sums(OpoSolver *s, double sums[3]);
/* n round trips like opo_run_round_trips, each followed by the FP64 tallies of that
 * round trip's output fields (tallies[3 k + f] = sum |A_f|^2 after round trip k, f = pump,
 * signal, idler; tallies may be NULL) and the reference's NaN probe (Solver3D.cuh:999-1005):
 * at the first round trip whose fields are not finite the loop stops and returns
 * OPO_ERR_NONFINITE.  *done (may be NULL) = round trips run.  One host synchronisation per
 * round trip (the reference also synchronises every round trip, for its probe). */
int opo_run_round_trips_tallied(OpoSolver *s, int n, double *tallies, int *done);

/* Per-pass device timing with CUDA events on the solver's stream.  While enabled,
 * passes are launched one by one (round trips are not replayed as graphs) with an event
 * pair around every pass kernel.  opo_pass_times() waits for the stream, returns the
 * accumulated milliseconds and launch counts per pass kind since the last call --
 * [0] t-pass, [1] x-pass or fused (x, y) plane pass, [2] y-pass, [3] other kernels --
 * and resets them.
 * No counterpart in the reference (its only timer is the wall clock, Common.cuh:74-90). */
int opo_set_pass_timing(OpoSolver *s, int enable);
int opo_pass_times(OpoSolver *s, double ms[4], long long counts[4]);

/* Time every compiled kernel variant (CTA size, first-stage radix) and tile size of
 * the t-, x- and y-passes on this solver's grid and keep the fastest for each, then
 * time the tuned x + y passes against every fused plane-pass variant (cluster size,
 * CTA size, first-stage radix) and keep the faster diffraction operator; results
 * are cached per (grid, precision, device) for the process, so later solvers of the same
 * shape reuse them without timing.  The candidates are timed on temporary scratch fields
 * (4 x nx ny nt complex values, allocated for the call), so the solver's own fields are
 * left as they were whether or not the cache held the grid.  Stands in for the
 * reference's compile-time block sizes (DtypesConsts.cuh:48-50). */
int opo_autotune(OpoSolver *s);

/* Pin the configuration instead of tuning it (same layout as opo_get_tuning).  Fails
 * with OPO_ERR_INVALID for a variant that is not compiled or a tile that cannot hold
 * the grid; the phase tables are rebuilt for the new FFT plans. */
int opo_set_tuning(OpoSolver *s, const int tuning[9]);

/* Chosen configuration: for the t-, x- and y-pass in turn, {CTA threads, tile elements
 * per field, first-stage radix}.  CTA threads 160 or 288 select the warp-specialised
 * kernels: 128 or 256 consumer threads plus one producer warp that streams the tiles
 * into a two-stage shared-memory ring with TMA (t- and y-passes in both precisions,
 * x-pass in FP64); batches run such a setting as its consumer CTA size.  A t-pass radix
 * with OPO_TUNE_LINE added (128 threads) selects the line-specialised t-pass: compiled
 * bodies for the time axes 64, 128 and 256, tiles of 8 FP32 pixels (two per packed
 * instruction) or 4 FP64 pixels; other grids (and the shipped Q2 launch grid) run the
 * generic kernel of the same size with the fallback radix (FP32: the given radix, FP64:
 * 4).  No counterpart in the reference. */
#define OPO_TUNE_LINE 256
int opo_get_tuning(const OpoSolver *s, int out[9]);

/* Diffraction operator as one fused plane pass (Solver3D.cuh:282-323 applied at :954 and
 * on the free-space return, :987-990): a thread-block cluster of `cluster` CTAs (2, 4 or
 * 8) per (field, t) plane holds the plane in its shared memory, applies the x factor to
 * its rows, exchanges through distributed shared memory and applies the y factor to its
 * columns, so the fields cross HBM once for both axes instead of twice.  cluster = 0
 * selects the separate x and y passes.  threads: 256 or 512; r1: first-stage radix of
 * both axes (4, 8 or 16; smaller when the plan needs it).  Fails with OPO_ERR_INVALID
 * when nx or ny is not a multiple of the cluster size or the slab does not fit; the
 * current configuration then stays.  Solvers start with a default plane pass where one
 * fits.  No counterpart in the reference (one cuFFT 3-D plan per field). */
int opo_set_plane_pass(OpoSolver *s, int cluster, int threads, int r1);
/* {cluster size (0: separate x and y passes), threads, first-stage radix}. */
int opo_get_plane_pass(const OpoSolver *s, int out[3]);

/* The CUDA stream (a cudaStream_t, returned as void*) on which this solver enqueues all
 * of its work, so that callers can order their own work or record timing events on it.
 * No counterpart in the reference (which runs on the legacy default stream). */
int opo_get_stream(const OpoSolver *s, void **stream);

/* Allocation-free FP64 tallies: the same three sums of |A|^2 as opo_field_sums, over
 * caller-owned device fields f0, f1, f2 of n complex values each (precision OPO_FP32 or
 * OPO_FP64), enqueued on `stream` (a cudaStream_t, or NULL for the legacy stream); the
 * call waits for the stream and writes the sums to host memory.  For callers that
 * cannot call cudaMalloc -- hosts whose own allocator has reserved the device memory,
 * or loops that cannot afford an allocation's implicit device synchronisation -- it
 * allocates nothing: its scratch is a fixed 24,600-byte device array inside the library,
 * held on every device that loads it until exit.  Limit: n <= 268,435,456 values per
 * field, larger n returns OPO_ERR_CAPACITY.  Non-finite sums return OPO_ERR_NONFINITE,
 * like opo_field_sums.  All calls share that array, so calls whose GPU work overlaps race
 * and must be ordered by the caller.  The first call on a device (and the first after the
 * device's context was reset) looks up the array's device address; make that first call
 * before any stream capture.  The result depends only on n (fixed summation order).
 * This entry point has no counterpart in the reference. */
int opo_field_sums_noalloc(const void *f0, const void *f1, const void *f2, size_t n, int precision,
                           void *stream, double sums[3]);
/* Message of the calling thread's last failed opo_field_sums_noalloc call ("" after a
 * successful one).  No counterpart in the reference. */
const char *opo_noalloc_last_error(void);

/* Measured FP64 arithmetic peak of the current device in TFLOP/s (independent FMA chains
 * on every SM, best of five event-timed launches; allocates a few bytes).  The reference
 * has no counterpart: it is the denominator of the t-pass's FP64-pipe roofline. */
int opo_fp64_peak(double *tflops);

/* Waits for the solver's stream.  OPO_ERR_CUDA when a warp-specialised pass gave up one
 * of its bounded pipeline waits: its tiles were not all written, so the fields are lost
 * and every call that reads or advances them fails until all four have been uploaded again
 * (opo_set_field) or initialised (opo_init_fields). */
int opo_synchronize(OpoSolver *s);
/* Bound of the warp-specialised passes' pipeline waits in SM clock cycles (0: the default,
 * about 2 s).  A short bound makes a pass give up and report OPO_ERR_CUDA instead of
 * waiting; it exists to exercise that error path.  The final drain of copies already
 * issued keeps the default bound.  No counterpart in the reference. */
int opo_set_wait_limit(OpoSolver *s, long long cycles);
int opo_round_trip_index(const OpoSolver *s);
/* Number of kernels this solver has launched since creation (graph nodes included). */
long long opo_kernel_launches(const OpoSolver *s);
const char *opo_last_error(const OpoSolver *s);
const char *opo_version(void);

/* ---- batched form: many instances, one persistent launch per pass ----------------- */

/* A batch advances every admitted instance (uneven grids and parameters, one slot
 * each) by whole cavity round trips, with one persistent kernel launch per pass for all
 * of them and each round trip replayed as one CUDA graph.  Instances are admitted while
 * their device memory fits the HBM budget; all instances of a batch take the same
 * number of z-steps.  The reference runs one instance per process (cuOPO3D.sh:65-86
 * sweeps by re-running the binary); this is the batched replacement of that loop.
 * tuning: {threads, tile elements, first-stage radix} for the t-, x- and y-pass
 * (opo_get_tuning layout), or NULL for the defaults. */
typedef struct OpoBatch OpoBatch;
int opo_batch_create(int precision, int capacity, size_t hbm_budget_bytes, const int tuning[9], OpoBatch **out);
void opo_batch_destroy(OpoBatch *b);
/* Admit one instance.  OPO_ERR_CAPACITY when no slot is free, when its fields and tables
 * (4 x nx ny nt complex values + 1 MiB) do not fit the budget left, or when the resident
 * instances take another number of z-steps (it fits once the batch has drained). */
int opo_batch_add(OpoBatch *b, const OpoParams *p, const double *w, int *slot);
int opo_batch_remove(OpoBatch *b, int slot);
int opo_batch_set_field(OpoBatch *b, int slot, int which, const void *src, int where, int elem_precision);
int opo_batch_get_field(OpoBatch *b, int slot, int which, void *dst, int where, int elem_precision);
/* Initialise a slot's fields on the device from its configuration: Api = Ap = the pump
 * of opo_pump_field, As = opo_noise(seed, sigma), Ai = 0 (or As when idler_copy). */
int opo_batch_init_fields(OpoBatch *b, int slot, const OpoConfig *cfg, uint64_t seed, double sigma, int idler_copy);
/* n round trips of every admitted instance (each continues its own round-trip count). */
int opo_batch_run_round_trips(OpoBatch *b, int n);
/* FP64 sums of |A|^2 of pump, signal, idler for every slot: sums[3 * slot + k]
 * (zero for empty slots); one batched reduction. */
int opo_batch_sums(OpoBatch *b, double *sums);
/* Slot info: {round trips done, round trips of its run, voxels, device bytes charged}. */
int opo_batch_info(const OpoBatch *b, int slot, long long out[4]);
/* Batch info: {admitted instances, bytes charged, budget, kernel launches}. */
int opo_batch_stats(const OpoBatch *b, long long out[4]);
int opo_batch_get_stream(const OpoBatch *b, void **stream);
int opo_batch_synchronize(OpoBatch *b);
const char *opo_batch_last_error(const OpoBatch *b);

/* ---- served form: continuous batching of sweep requests --------------------------- */

typedef struct OpoServeRequest {
    OpoConfig cfg;        /* the instance; cfg.total_rt bounds its round trips           */
    double arrival_s;     /* arrival time after the start of the stream                   */
    uint64_t seed;        /* signal noise seed (opo_noise)                                */
    double noise_sigma;   /* signal noise standard deviation per component                */
    double tol;           /* retire when |dPs/Ps| over one round trip <= tol (<= 0: never) */
    double *out_fields[3];/* optional host buffers (nx ny nt complex128 each, [t][y][x]) that
                             receive the final pump, signal and idler at retirement; NULL
                             entries are skipped                                          */
} OpoServeRequest;

typedef struct OpoServeOptions {
    int precision;        /* OPO_FP32 / OPO_FP64 for every request                        */
    int capacity;         /* slots (resident instances at most)                           */
    size_t hbm_budget;    /* device bytes the resident instances may take                 */
    int realtime;         /* 1: admit a request only once the wall clock reaches its arrival */
    int tuning_set;       /* 1: use `tuning` for the batch kernels                        */
    int tuning[9];
} OpoServeOptions;

typedef struct OpoServeResult {
    int status;           /* OPO_OK, OPO_ERR_NONFINITE (fields stopped being finite),
                             OPO_ERR_INVALID (malformed), OPO_ERR_CAPACITY (does not fit
                             even with nothing else resident)                              */
    int round_trips;
    double admit_s, done_s, latency_s;  /* latency = done - arrival                        */
    double power[3];      /* final FP64 sums of |A|^2 (pump, signal, idler)              */
    long long voxel_steps;
} OpoServeResult;

/* Run a stream of requests with continuous batching (see serve.cpp): requests that
 * arrive while others run are admitted as slots and memory free up, and all resident
 * instances advance together one round trip at a time.  stats = {p50 latency s, p99
 * latency s, wall s, voxel-steps/s, most resident at once, kernel launches, voxel-steps,
 * completed}.  The reference's sweep re-runs its binary per point (cuOPO3D.sh:65-86). */
int opo_serve(const OpoServeRequest *reqs, int n, const OpoServeOptions *opt, OpoServeResult *out, double stats[8]);

/* ---- output files (see writer.cpp) -------------------------------------------------- */

enum { OPO_FILES_TEXT = 0, OPO_FILES_BINARY = 1 };
/* Writes field `which` (OPO_FIELD_*) with one device-to-host copy.  OPO_FILES_TEXT: the
 * reference's text dumps (Files.cuh:73-211 as cuOPO3D.cu:75-85 calls them), 20 significant
 * digits, "_r.dat" / "_i.dat" pairs: for every t, "<slice_prefix><t>" holds the (x, y) slice
 * as NY rows of NX tab-terminated values (saveMatrixComplex_TimeSlice); for every pixel,
 * "<trace_prefix><x>_y_<y>" holds its NT values one per line (SaveElectricField_time3D_GPU;
 * main passes "As_temporal_x_" as the prefix).  Either prefix may be NULL to skip that set.
 * OPO_FILES_BINARY: one file "<slice_prefix>.bin": a 32-byte header ("OPO3DFLD", then int32
 * version 1, nx, ny, nt, bytes per complex value, which) and the field [t][y][x] in the
 * solver's precision.  Files are written by up to 16 host threads. */
int opo_save_fields(OpoSolver *s, int which, const char *slice_prefix, const char *trace_prefix, int format);

/* ---- threshold sweeps (see sweep.cpp) ---------------------------------------------- */

/* The reference's scan over pump power and waist (cuOPO3D.sh:58-80 runs the binary once
 * per point; the threshold pairs are appended by saveAppendedValues2Columns, Files.cuh:
 * 215-233, called at cuOPO3D.cu:88), run as waves of instances on one OpoBatch. */
typedef struct OpoSweepOptions {
    int precision;        /* OPO_FP32 / OPO_FP64                                          */
    int round_trips;      /* round trips per point                                        */
    int window;           /* the gain is measured over the last `window` round trips      */
    uint64_t seed;        /* signal noise seed of point k: seed + k (opo_noise)           */
    double noise_sigma;   /* signal noise standard deviation per component                */
    size_t hbm_budget;    /* device bytes the resident points may take                    */
    int capacity;         /* points resident at once (<= 0: all)                          */
    int tuning_set;       /* 1: use `tuning` for the batch kernels                        */
    int tuning[9];
} OpoSweepOptions;

typedef struct OpoSweepPoint {
    double P, w0;         /* in: pump power (W) and waist (um) of the point               */
    int status;           /* out: OPO_OK, OPO_ERR_NONFINITE (stopped at that round trip),
                             OPO_ERR_INVALID / OPO_ERR_CAPACITY (not run)                 */
    int round_trips;      /* out: round trips run                                         */
    double sums[3];       /* out: final FP64 sums |A|^2 of pump, signal, idler            */
    double power_xy[3];   /* out: the reference's averagePowerCutXY of each (opo_power_cut_xy) */
    double output_power;  /* out: power_xy[signal] x (1 - Rs), the output-coupled signal  */
    double gain;          /* out: signal round-trip gain (Ps(n) / Ps(n - window))^(1/window) */
    int above;            /* out: 1 when gain > 1 (above threshold)                       */
} OpoSweepPoint;

/* Run every point of base with its (P, w0) for opt->round_trips round trips.  tallies (may
 * be NULL): n x round_trips x 3 FP64 sums, tallies[(k R + r) 3 + f] after round trip r + 1
 * of point k (NaN after a point stopped). */
int opo_sweep(const OpoConfig *base, OpoSweepPoint *pts, int n, const OpoSweepOptions *opt, double *tallies);
/* Threshold bracket of run points (one waist): the largest P below threshold that is under
 * the smallest P above it, and the power where ln(gain), linear between them, crosses 0.
 * OPO_ERR_INVALID when the scan does not cross threshold. */
int opo_sweep_threshold(const OpoSweepPoint *pts, int n, double *p_below, double *p_above, double *p_est);
/* Writes "P <tab> output_power" per completed point in the format of the reference's
 * saveAppendedValues2Columns (default stream formatting; append or truncate). */
int opo_sweep_write(const char *path, const OpoSweepPoint *pts, int n, int append);

#ifdef __cplusplus
}
#endif
#endif /* CUOPO3D_H */
