// Test infrastructure only (never linked into the product): a driver that builds the
// reference cuOPO3D solver from its own, unmodified headers (src/headers of
// alfredos84/cuOPO3D) for one grid / precision / fix set, runs it, and dumps the
// derived scalars and the fields so that the CPU oracle can be pinned against the
// reference and the reference's cuFFT pipeline can be timed on the same GPU.
//
// Compile-time knobs (the reference's grid is compile-time, DtypesConsts.cuh:30-54):
//   RH_NX RH_NY RH_NT RH_NZ RH_NRT  grid, slices and round trips
//   RH_FP64  1: real_t=double, complex_t=cufftDoubleComplex, Z2Z transforms and double
//               math (the "ref-fixed-fp64" parity build); 0: the shipped FP32 types
//   RH_FIX   1: replace the three members whose shipped behaviour is broken or
//               non-deterministic (Solver3D.cuh:572-639 dispersion launch grid and
//               scale, :644-694 GDD transform of an unwritten buffer, :726-788
//               diffraction scale 1/SIZE) with minimally corrected versions that
//               call the reference's own kernels; 0: everything as shipped.
//
// The reference's DtypesConsts.cuh is skipped by pre-defining its include guard; this
// file supplies the same names (types, grid constants, physical constants) instead.

#include "Libraries.cuh"

#define _DTYPESCONSTSCUH

#if RH_FP64
using real_t = double;
using complex_t = cufftDoubleComplex;
#define cufftExecC2C cufftExecZ2Z
#define CUFFT_C2C CUFFT_Z2Z
#define cosf cos
#define sinf sin
#define expf exp
#define powf pow
#define sqrtf sqrt
#define logf log
#define make_float2 make_double2
#define make_cuFloatComplex make_cuDoubleComplex
#else
using real_t = float;
using complex_t = cufftComplex;
#endif
using rVech_t = thrust::host_vector<real_t>;
using rVecd_t = thrust::device_vector<real_t>;
using cVech_t = thrust::host_vector<complex_t>;
using cVecd_t = thrust::device_vector<complex_t>;

const uint32_t NX = RH_NX;
const uint32_t NY = RH_NY;
const uint32_t NT = RH_NT;
const uint32_t SIZE = NX * NY * NT;
const uint32_t NZ = RH_NZ;
const uint32_t BLKT = 1 << 5;
const uint32_t BLKX = 1 << 4;
const uint32_t BLKY = BLKX;
const uint32_t NRT = RH_NRT;
const real_t PI = 3.14159265358979323846;
const real_t C = 299792458 * 1E6 / 1E12;
const real_t EPS0 = 8.8541878128E-12 * 1E12 / 1E6;
const size_t nBytes1Dr = sizeof(real_t) * NT;
const size_t nBytes1Dc = sizeof(complex_t) * NT;
const size_t nBytes2Dr = sizeof(real_t) * NX * NY;
const size_t nBytes2Dc = sizeof(complex_t) * NX * NY;
const size_t nBytes3Dr = sizeof(real_t) * SIZE;
const size_t nBytes3Dc = sizeof(complex_t) * SIZE;

#include "PackageLibraries.cuh"

#include <map>
#include <sstream>
#include <vector>

#if RH_FIX
// Scale kernel used by the corrected members: every voxel of three fields times s.
__global__ void rhScale3(complex_t *a, complex_t *b, complex_t *c, real_t s, uint32_t n)
{
    uint32_t i = threadIdx.x + blockDim.x * blockIdx.x;
    if (i < n) {
        a[i].x *= s; a[i].y *= s;
        if (b) { b[i].x *= s; b[i].y *= s; }
        if (c) { c[i].x *= s; c[i].y *= s; }
    }
}

static inline dim3 rhGrid2D() { return dim3((NX + BLKX - 1) / BLKX, (NY + BLKY - 1) / BLKY); }
static inline dim3 rhBlock2D() { return dim3(BLKX, BLKY); }
static inline dim3 rhGrid1D() { return dim3((SIZE + 255) / 256); }

// Corrected dispersion (reference Solver3D.cuh:572-639): the transposes, the product and
// the scale cover every pixel (the shipped <<<64,64>>> launches touch only y=0), and
// the inverse transform is normalised by 1/NT instead of 1/SIZE.
#define RH_FIXED_MEMBERS(CR)                                                               \
template<> void Solver<CR>::dispersion()                                                   \
{                                                                                          \
    cufftHandle plan; int n = NT;                                                          \
    cufftPlanMany(&plan, 1, &n, nullptr, 1, NT, nullptr, 1, NT, CUFFT_C2C, NX * NY);       \
    complex_t *p = thrust::raw_pointer_cast(A->Ap.data());                                 \
    complex_t *s = thrust::raw_pointer_cast(A->As.data());                                 \
    complex_t *i = thrust::raw_pointer_cast(A->Ai.data());                                 \
    complex_t *lp = thrust::raw_pointer_cast(A->eiLz_p.data());                            \
    complex_t *ls = thrust::raw_pointer_cast(A->eiLz_s.data());                            \
    complex_t *li = thrust::raw_pointer_cast(A->eiLz_i.data());                            \
    complex_t *buf[9];                                                                     \
    for (int k = 0; k < 9; k++) CHECK(cudaMalloc((void **)&buf[k], nBytes3Dc));            \
    tensor3D_to_2D_3Fileds<<<rhGrid2D(), rhBlock2D()>>>(buf[0], p, buf[1], s, buf[2], i);  \
    CHECK(cudaDeviceSynchronize());                                                        \
    for (int k = 0; k < 3; k++) cufftExecC2C(plan, buf[k], buf[3 + k], CUFFT_INVERSE);     \
    CHECK(cudaDeviceSynchronize());                                                        \
    rhScale3<<<rhGrid1D(), 256>>>(buf[3], buf[4], buf[5], real_t(1) / real_t(NT), SIZE);   \
    CHECK(cudaDeviceSynchronize());                                                        \
    kernelDispersionPropagatorProduct<<<rhGrid2D(), rhBlock2D()>>>(                        \
        buf[6], buf[3], lp, buf[7], buf[4], ls, buf[8], buf[5], li);                       \
    CHECK(cudaDeviceSynchronize());                                                        \
    for (int k = 0; k < 3; k++) cufftExecC2C(plan, buf[6 + k], buf[k], CUFFT_FORWARD);     \
    CHECK(cudaDeviceSynchronize());                                                        \
    tensor2D_to_3D_3Fileds<<<rhGrid2D(), rhBlock2D()>>>(p, buf[0], s, buf[1], i, buf[2]);  \
    CHECK(cudaDeviceSynchronize());                                                        \
    for (int k = 0; k < 9; k++) CHECK(cudaFree(buf[k]));                                   \
    cufftDestroy(plan);                                                                    \
}                                                                                          \
template<> void Solver<CR>::GDDCompensation(cVecd_t &Ax)                                   \
{                                                                                          \
    if (!Cav->gdd) return;                                                                 \
    cufftHandle plan; int n = NT;                                                          \
    cufftPlanMany(&plan, 1, &n, nullptr, 1, NT, nullptr, 1, NT, CUFFT_C2C, NX * NY);       \
    complex_t *a = thrust::raw_pointer_cast(Ax.data());                                    \
    real_t *w = thrust::raw_pointer_cast(A->w.data());                                     \
    complex_t *aux, *tx, *wx;                                                              \
    CHECK(cudaMalloc((void **)&aux, nBytes3Dc));                                           \
    CHECK(cudaMalloc((void **)&tx, nBytes3Dc));                                            \
    CHECK(cudaMalloc((void **)&wx, nBytes3Dc));                                            \
    tensor3D_to_2D<<<rhGrid2D(), rhBlock2D()>>>(tx, a);                                    \
    CHECK(cudaDeviceSynchronize());                                                        \
    cufftExecC2C(plan, tx, wx, CUFFT_INVERSE);                                             \
    CHECK(cudaDeviceSynchronize());                                                        \
    rhScale3<<<rhGrid1D(), 256>>>(wx, nullptr, nullptr, real_t(1) / real_t(NT), SIZE);     \
    CHECK(cudaDeviceSynchronize());                                                        \
    real_t GDD = -(Cav->gamma) * (Cr->b2s) * (Cr->Lcr);                                    \
    kernelGDDCompensation<<<rhGrid2D(), rhBlock2D()>>>(wx, aux, w, GDD);                   \
    CHECK(cudaDeviceSynchronize());                                                        \
    cufftExecC2C(plan, wx, tx, CUFFT_FORWARD);                                             \
    CHECK(cudaDeviceSynchronize());                                                        \
    tensor2D_to_3D<<<rhGrid2D(), rhBlock2D()>>>(a, tx);                                    \
    CHECK(cudaDeviceSynchronize());                                                        \
    CHECK(cudaFree(aux)); CHECK(cudaFree(tx)); CHECK(cudaFree(wx));                        \
    cufftDestroy(plan);                                                                    \
}                                                                                          \
template<> void Solver<CR>::diffractionInCrystal()                                         \
{                                                                                          \
    cufftHandle plan; int n[2] = {(int)NY, (int)NX}; int emb[2] = {(int)NY, (int)NX};      \
    cufftPlanMany(&plan, 2, n, emb, 1, NX * NY, emb, 1, NX * NY, CUFFT_C2C, NT);           \
    complex_t *f[3] = {thrust::raw_pointer_cast(A->Ap.data()),                             \
                       thrust::raw_pointer_cast(A->As.data()),                             \
                       thrust::raw_pointer_cast(A->Ai.data())};                            \
    complex_t *q[3] = {thrust::raw_pointer_cast(A->AQp.data()),                            \
                       thrust::raw_pointer_cast(A->AQs.data()),                            \
                       thrust::raw_pointer_cast(A->AQi.data())};                           \
    complex_t *e[3] = {thrust::raw_pointer_cast(A->eiQz_p.data()),                         \
                       thrust::raw_pointer_cast(A->eiQz_s.data()),                         \
                       thrust::raw_pointer_cast(A->eiQz_i.data())};                        \
    complex_t *aux[3];                                                                     \
    for (int k = 0; k < 3; k++) CHECK(cudaMalloc((void **)&aux[k], nBytes3Dc));            \
    for (int k = 0; k < 3; k++) cufftExecC2C(plan, f[k], q[k], CUFFT_FORWARD);             \
    CHECK(cudaDeviceSynchronize());                                                        \
    kernelDiffractionPropagatorProduct<<<rhGrid2D(), rhBlock2D()>>>(                       \
        aux[0], e[0], q[0], aux[1], e[1], q[1], aux[2], e[2], q[2]);                       \
    CHECK(cudaDeviceSynchronize());                                                        \
    for (int k = 0; k < 3; k++) cufftExecC2C(plan, aux[k], f[k], CUFFT_INVERSE);           \
    CHECK(cudaDeviceSynchronize());                                                        \
    rhScale3<<<rhGrid1D(), 256>>>(f[0], f[1], f[2], real_t(1) / real_t(NX * NY), SIZE);    \
    CHECK(cudaDeviceSynchronize());                                                        \
    for (int k = 0; k < 3; k++) CHECK(cudaFree(aux[k]));                                   \
    cufftDestroy(plan);                                                                    \
}

RH_FIXED_MEMBERS(PPLN)
RH_FIXED_MEMBERS(MgOsPPLT)
#endif

// ---------------------------------------------------------------------------------
// Driver.  Arguments are key=value pairs (see usage()).

typedef std::map<std::string, std::string> Args;

static double argd(const Args &a, const char *k, double def)
{
    auto it = a.find(k);
    return it == a.end() ? def : atof(it->second.c_str());
}
static std::string args(const Args &a, const char *k, const char *def)
{
    auto it = a.find(k);
    return it == a.end() ? std::string(def) : it->second;
}

static void readField(const std::string &path, cVecd_t &dst)
{
    // Raw little-endian complex128, SIZE elements, layout [t][y][x].
    std::vector<double> buf(2 * (size_t)SIZE);
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) { fprintf(stderr, "cannot open %s\n", path.c_str()); exit(2); }
    size_t got = fread(buf.data(), sizeof(double), buf.size(), fp);
    fclose(fp);
    if (got != buf.size()) { fprintf(stderr, "short read %s\n", path.c_str()); exit(2); }
    cVech_t h(SIZE);
    for (size_t i = 0; i < SIZE; i++) { h[i].x = (real_t)buf[2 * i]; h[i].y = (real_t)buf[2 * i + 1]; }
    thrust::copy(h.begin(), h.end(), dst.begin());
}

static void writeField(const std::string &path, const cVecd_t &src)
{
    cVech_t h = src;
    std::vector<double> buf(2 * h.size());
    for (size_t i = 0; i < h.size(); i++) { buf[2 * i] = h[i].x; buf[2 * i + 1] = h[i].y; }
    FILE *fp = fopen(path.c_str(), "wb");
    fwrite(buf.data(), sizeof(double), buf.size(), fp);
    fclose(fp);
}

static void writeReal(const std::string &path, const rVecd_t &src)
{
    rVech_t h = src;
    std::vector<double> buf(h.begin(), h.end());
    FILE *fp = fopen(path.c_str(), "wb");
    fwrite(buf.data(), sizeof(double), buf.size(), fp);
    fclose(fp);
}

template <typename Crystal>
static int run(const Args &a)
{
    const std::string mode = args(a, "mode", "single");
    const std::string out = args(a, "out", "ref");
    real_t LX = argd(a, "LX", 400), LY = argd(a, "LY", 400), Lcr = argd(a, "Lcr", 5000);
    real_t T = argd(a, "T", 27), Lambda = argd(a, "Lambda", 6.97);
    real_t lp = argd(a, "lp", 0.532);
    real_t ls = argd(a, "ls", 2 * lp);
    real_t li = ls * lp / (ls - lp);
    Crystal *cr = new Crystal(LX, LY, Lcr, T, Lambda, lp, ls, li);
    if (a.count("dQ")) cr->dQ = argd(a, "dQ", 0);
    if (a.count("alpha_p")) cr->alpha_crp = argd(a, "alpha_p", 0);
    if (a.count("alpha_s")) cr->alpha_crs = argd(a, "alpha_s", 0);
    if (a.count("alpha_i")) cr->alpha_cri = argd(a, "alpha_i", 0);

    real_t Lcav = argd(a, "Lcav", 4 * cr->Lcr), Rs = argd(a, "Rs", 0.98), Ri = argd(a, "Ri", Rs);
    Cavity<Crystal> *cav = new Cavity<Crystal>(cr, Lcav, Rs, Ri);
    cav->gdd = false;
    cav->gamma = 0;
    if (argd(a, "gdd", 0) != 0) cav->setGDDCompensation(argd(a, "gdd", 0));

    real_t P = argd(a, "P", 1), FWHM = argd(a, "FWHM", 2), w0 = argd(a, "w0", 50);
    real_t focal = argd(a, "focal", Lcr / 2);
    EFields<Crystal> *A = new EFields<Crystal>(lp, ls, li, P, w0, cr);
    A->resFields = std::make_tuple(false, true, true);
    if (a.count("resonant")) {
        // bit mask of resonant fields (1 pump, 2 signal, 4 idler), default signal + idler as main()
        const int r = (int)argd(a, "resonant", 6);
        A->resFields = std::make_tuple((r & 1) != 0, (r & 2) != 0, (r & 4) != 0);
    }
    real_t twin = argd(a, "twin", 0);
    A->setTimeFreqVectors(twin > 0 ? twin : cav->trt);
    A->setPumpField(P, FWHM, w0, focal, args(a, "pump", "focused-pulsed"));
    A->Ap = A->Api;
    if (a.count("init_s")) readField(args(a, "init_s", ""), A->As);
    else thrust::fill(A->As.begin(), A->As.end(), complex_t{0, 0});
    if (a.count("init_i")) readField(args(a, "init_i", ""), A->Ai);
    else thrust::fill(A->Ai.begin(), A->Ai.end(), complex_t{0, 0});

    Solver<Crystal> *solv = new Solver<Crystal>(cr, cav, A);

    // Number of z-steps the reference's float loop takes (Solver3D.cuh:949).
    int nsteps = 0;
    for (real_t z = 0; z <= cr->Lcr; z += (cr->dz)) nsteps++;

    if (mode == "single" || mode == "opo") {
        if (mode == "single") {
            solv->setDispersionPropagators();
            solv->setDiffractionPropagators();
            solv->runSinglePass();
        } else {
            solv->runOPO();
        }
        CHECK(cudaDeviceSynchronize());
        writeField(out + "_Ap.bin", A->Ap);
        writeField(out + "_As.bin", A->As);
        writeField(out + "_Ai.bin", A->Ai);
        writeField(out + "_Api.bin", A->Api);
        writeReal(out + "_t.bin", A->t);
        writeReal(out + "_w.bin", A->w);
        FILE *fp = fopen((out + "_scalars.txt").c_str(), "w");
#define RH_PUT(name, val) fprintf(fp, "%s %.17g\n", name, (double)(val))
        RH_PUT("np", cr->np); RH_PUT("ns", cr->ns); RH_PUT("ni", cr->ni);
        RH_PUT("vp", cr->vp); RH_PUT("vs", cr->vs); RH_PUT("vi", cr->vi);
        RH_PUT("b2p", cr->b2p); RH_PUT("b2s", cr->b2s); RH_PUT("b2i", cr->b2i);
        RH_PUT("b3p", cr->b3p); RH_PUT("b3s", cr->b3s); RH_PUT("b3i", cr->b3i);
        RH_PUT("dQ", cr->dQ); RH_PUT("dk", cr->dk);
        RH_PUT("dx", cr->dx); RH_PUT("dy", cr->dy); RH_PUT("dz", cr->dz);
        RH_PUT("kp", A->kp); RH_PUT("ks", A->ks); RH_PUT("ki", A->ki);
        RH_PUT("kappa_p", A->kappa_p); RH_PUT("kappa_s", A->kappa_s); RH_PUT("kappa_i", A->kappa_i);
        RH_PUT("trt", cav->trt); RH_PUT("dt", cav->dt);
        RH_PUT("nsteps", nsteps); RH_PUT("NX", NX); RH_PUT("NY", NY); RH_PUT("NT", NT);
        RH_PUT("NZ", NZ); RH_PUT("NRT", NRT); RH_PUT("fp64", RH_FP64); RH_PUT("fix", RH_FIX);
        RH_PUT("power_cut_xy_As", solv->averagePowerCutXY(A->As));
#undef RH_PUT
        fclose(fp);
        printf("RH_DONE nsteps=%d\n", nsteps);
        return 0;
    }

    // Timing: each step is one cavity round trip made of the reference's public
    // members in the order of Solver3D.cuh:981-997 (fresh pump, propagators, SSFM,
    // free-space return, GDD, mirrors).
    if (mode == "time_opo") {
        int warm = (int)argd(a, "warmup", 1), steps = (int)argd(a, "steps", 2);
        solv->setDispersionPropagators();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0); cudaEventCreate(&e1);
        float total_ms = 0;
        std::vector<float> per;
        for (int k = 0; k < warm + steps; k++) {
            CHECK(cudaDeviceSynchronize());
            cudaEventRecord(e0);
            A->Ap = A->Api;
            solv->setDiffractionPropagators();
            solv->SSFM();
            solv->setDiffractionPropagatorsInFreeSpace(cr->Lcr);
            solv->diffractionInFreeSpace();
            if (cav->gdd) { solv->GDDCompensation(A->As); solv->GDDCompensation(A->Ai); }
            if (std::get<1>(A->resFields)) cav->applyReflectivity(A->As, cav->Rs, 0.0f);
            if (std::get<2>(A->resFields)) cav->applyReflectivity(A->Ai, cav->Ri, 0.0f);
            cudaEventRecord(e1);
            CHECK(cudaEventSynchronize(e1));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (k >= warm) { total_ms += ms; per.push_back(ms); }
        }
        double vs = (double)SIZE * nsteps * steps / (total_ms * 1e-3);
        printf("{\"rh_time_opo\": true, \"voxel_steps_per_s\": %.6e, \"ms_per_round_trip\": %.4f, "
               "\"nsteps\": %d, \"steps\": %d, \"warmup\": %d, \"NX\": %u, \"NY\": %u, \"NT\": %u, "
               "\"fp64\": %d, \"fix\": %d}\n",
               vs, total_ms / steps, nsteps, steps, warm, NX, NY, NT, RH_FP64, RH_FIX);
        return 0;
    }
    fprintf(stderr, "unknown mode %s\n", mode.c_str());
    return 2;
}

int main(int argc, char **argv)
{
    Args a;
    for (int k = 1; k < argc; k++) {
        std::string s(argv[k]);
        size_t eq = s.find('=');
        if (eq == std::string::npos) { fprintf(stderr, "bad arg %s\n", argv[k]); return 2; }
        a[s.substr(0, eq)] = s.substr(eq + 1);
    }
    std::string crystal = args(a, "crystal", "ppln");
    if (crystal == "ppln") return run<PPLN>(a);
    if (crystal == "mgosplt") return run<MgOsPPLT>(a);
    fprintf(stderr, "unknown crystal %s\n", crystal.c_str());
    return 2;
}
