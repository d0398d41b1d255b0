// Host side of the solver: FP64 physics of the reference classes (crystal, fields,
// cavity), FFT stage plans, phase tables, the pass schedule of a single pass and of a
// cavity round trip (captured as CUDA graphs), and the C-ABI of include/cuopo3d.h.

#include "../../include/cuopo3d.h"
#include "fft_gain.h"
#include "opo_internal.h"
#include "solver_internal.h"

#include <cudaTypedefs.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <new>
#include <string>
#include <vector>

namespace {

using cd = std::complex<double>;

// Physical constants of the reference, DtypesConsts.cuh:55-57.
constexpr double kPi = 3.14159265358979323846;
constexpr double kC = 299792458 * 1E6 / 1E12;           // um / ps
constexpr double kEps0 = 8.8541878128E-12 * 1E12 / 1E6; // W ps / (V^2 um)

// ---------------------------------------------------------------------------------
// Sellmeier models.  Both reference crystals share one form
//   n^2 = a0 + sum_r B_r / (L^2 - C_r^2) + d L^2,
// (PPLN.cuh:97-117 with temperature-dependent B, C; MgOsPPLT.cuh:96-112), so that
//   res_p(L) = sum_r B_r / (L^2 - C_r^2)^p,  R2 = res_2 - d,
//   dn/dl = -L R2 / n, and the higher derivatives / GV / GVD / TOD follow the
// reference expressions (PPLN.cuh:149-259, MgOsPPLT.cuh:138-226).
struct Sellmeier {
    double a0, d;
    int nr;
    double B[3], C2[3];  // C2 = C_r^2

    double n(double L) const
    {
        double v = a0 + d * L * L;
        for (int r = 0; r < nr; r++) v += B[r] / (L * L - C2[r]);
        return std::sqrt(v);
    }
    double res(double L, int p) const
    {
        double v = 0;
        for (int r = 0; r < nr; r++) v += B[r] / std::pow(L * L - C2[r], p);
        return v;
    }
    double R2(double L) const { return res(L, 2) - d; }
    double dn(double L) const { return -L * R2(L) / n(L); }
    double d2n(double L) const
    {
        const double nn = n(L);
        return (L * dn(L) / (nn * nn) - 1 / nn) * R2(L) + 4 * L * L / nn * res(L, 3);
    }
    double d3n(double L) const
    {
        const double nn = n(L), d1 = dn(L), d2 = d2n(L);
        const double AA = ((2 * d1 + L * d2) / (nn * nn) - 2 * L * d1 * d1 / (nn * nn * nn)) * R2(L);
        const double BB = (12 * L / nn - 4 * L * L / nn * d2 * (1 - 1 / nn)) * res(L, 3);
        const double CC = -24 * L * L * L / nn * res(L, 4);
        return AA + BB + CC;
    }
    // The exact third derivative: differentiating n n'' = -R2 + 4 L^2 res_3 - n'^2 once
    // more gives n''' = (12 L res_3 - 24 L^3 res_4 - 3 n' n'') / n.  (d3n above is the
    // reference's expression, which differs from it; the reference only prints its TOD.)
    double d3n_exact(double L) const
    {
        const double nn = n(L);
        return (12 * L * res(L, 3) - 24 * L * L * L * res(L, 4) - 3 * dn(L) * d2n(L)) / nn;
    }
    double vg(double L) const { return kC / (n(L) - L * dn(L)); }
    double gvd(double L) const { return std::pow(L, 3) * d2n(L) / (2 * kPi * kC * kC); }
    double tod_of(double L, double d3) const
    {
        return -std::pow(L, 4) / (4 * kPi * kPi * kC * kC * kC) * (3 * d2n(L) + L * d3);
    }
    double tod(double L) const { return tod_of(L, d3n(L)); }              // as the reference prints it
    double tod_exact(double L) const { return tod_of(L, d3n_exact(L)); }  // applied with OPO_TOD
};

struct CrystalModel {
    Sellmeier s[3];  // pump, signal, idler (polarisation-dependent crystals differ)
    double d33;
    double alpha[3];
    bool qpm;        // quasi-phase matched: dk includes the grating term 2 pi / Lambda
};

// One index model of a crystal: `extraordinary` selects the polarisation of crystals
// that have two (ZGP); the QPM crystals are extraordinary-only.
bool sellmeier_of(int kind, double T, bool extraordinary, Sellmeier &m)
{
    if (kind == OPO_PPLN || kind == OPO_MGOPPLN) {
        // n^2 = G1 + G2/(L^2 - G3^2) + G4/(L^2 - a5^2) - a6 L^2 with Gi = ai + bi f,
        // f = (T - 24.5)(T + 570.82): Jundt for congruent LiNbO3 (PPLN.cuh:100-115), Gayer
        // for MgO:LiNbO3 (MgOPPLN.cuh:99-117)
        const bool mgo = kind == OPO_MGOPPLN;
        const double f = (T - 24.5) * (T + 570.82);
        const double a1 = mgo ? 5.756 : 5.35583, a2 = mgo ? 0.0983 : 0.100473, a3 = mgo ? 0.2020 : 0.20692,
                     a4 = mgo ? 189.32 : 100.0, a5 = mgo ? 12.52 : 11.34927, a6 = mgo ? 1.32e-2 : 1.5334e-2,
                     b1 = mgo ? 2.860e-6 : 4.629e-7, b2 = mgo ? 4.700e-8 : 3.862e-8,
                     b3 = mgo ? 6.113e-8 : -0.89e-8, b4 = mgo ? 1.516e-4 : 2.657e-5;
        const double G3 = a3 + b3 * f;
        m.a0 = a1 + b1 * f;
        m.d = -a6;
        m.nr = 2;
        m.B[0] = a2 + b2 * f; m.C2[0] = G3 * G3;
        m.B[1] = a4 + b4 * f; m.C2[1] = a5 * a5;
        return true;
    }
    if (kind == OPO_MGOSPPLT) {
        // Bruner, stoichiometric LiTaO3 (MgOsPPLT.cuh:99-110)
        const double TK2 = std::pow(T + 273.15, 2);
        const double Cc = 0.185087 + 1.607839e-8 * TK2;
        m.a0 = 4.502483;
        m.d = -0.02357;
        m.nr = 3;
        m.B[0] = 0.007294 + 3.483933e-8 * TK2; m.C2[0] = Cc * Cc;
        m.B[1] = 0.073423;                     m.C2[1] = 0.199595 * 0.199595;
        m.B[2] = 0.001;                        m.C2[2] = 7.99724 * 7.99724;
        return true;
    }
    if (kind == OPO_ZGP) {
        // Zelmon, ZnGeP2 (ZGP.cuh:103-126): n^2 = A + B L^2/(L^2 - CC) + D L^2/(L^2 - E),
        // i.e. (A + B + D) + B CC/(L^2 - CC) + D E/(L^2 - E); no temperature dependence
        const double A = extraordinary ? 8.0929 : 8.0409, B = extraordinary ? 1.8649 : 1.68625,
                     CC = extraordinary ? 0.41468 : 0.40824, D = extraordinary ? 0.84052 : 1.2880,
                     E = extraordinary ? 452.05 : 611.05;
        m.a0 = A + B + D;
        m.d = 0;
        m.nr = 2;
        m.B[0] = B * CC; m.C2[0] = CC;
        m.B[1] = D * E;  m.C2[1] = E;
        return true;
    }
    return false;
}

// pol: bit f set = wave f (pump, signal, idler) extraordinary (used by ZGP only).
bool crystal_model(int kind, double T, unsigned pol, CrystalModel &m)
{
    for (int f = 0; f < 3; f++)
        if (!sellmeier_of(kind, T, (pol >> f) & 1u, m.s[f])) return false;
    switch (kind) {
    case OPO_PPLN:      // PPLN.cuh:57-60
    case OPO_MGOPPLN:   // MgOPPLN.cuh:57-60
        m.d33 = 25.20e-6;
        m.alpha[0] = 0.025e-4; m.alpha[1] = 0.002e-4; m.alpha[2] = 0.002e-4;
        m.qpm = true;
        break;
    case OPO_MGOSPPLT:  // MgOsPPLT.cuh:57-60
        m.d33 = 11.0e-6;
        m.alpha[0] = 1.57e-4; m.alpha[1] = 0.17e-6; m.alpha[2] = 0.17e-6;
        m.qpm = true;
        break;
    default:            // ZGP.cuh:55-58: birefringent phase matching, no grating
        m.d33 = 75.0e-6;
        m.alpha[0] = 1.57e-4; m.alpha[1] = 0.17e-6; m.alpha[2] = 0.17e-6;
        m.qpm = false;
        break;
    }
    return true;
}

// Step count of the reference loop `for (real_t z = 0; z <= Lcr; z += dz)`
// (Solver3D.cuh:949) in FP32 or FP64.
int zloop_steps(double Lcr, double dz, bool f32)
{
    int n = 0;
    if (f32) {
        const float L = (float)Lcr, d = (float)dz;
        for (float z = 0; z <= L; z += d) n++;
    } else {
        for (double z = 0; z <= Lcr; z += dz) n++;
    }
    return n;
}

// ---------------------------------------------------------------------------------
// FFT stage plans and tables.

opo::FastDiv make_fastdiv(unsigned d)
{
    opo::FastDiv f{d ? d : 1u, 0u, 0u};
    unsigned l = 0;
    while ((1ull << l) < f.d) l++;
    if ((1ull << l) == f.d) {
        f.s = l;
        return f;
    }
    f.m = (unsigned)(((1ull << (31 + l)) + f.d - 1) / f.d);
    f.s = l - 1;
    return f;
}

// Radices for 2^e, each <= rmax, largest first and balanced.
bool split_pow2(int e, int rmax, std::vector<int> &out)
{
    static const int t16[][3] = {{0, 0, 0}, {2, 0, 0}, {4, 0, 0}, {8, 0, 0}, {16, 0, 0}, {8, 4, 0},
                                 {8, 8, 0}, {16, 8, 0}, {16, 16, 0}, {8, 8, 8}, {16, 8, 8}, {16, 16, 8},
                                 {16, 16, 16}};
    static const int t8[][4] = {{0, 0, 0, 0}, {2, 0, 0, 0}, {4, 0, 0, 0}, {8, 0, 0, 0}, {4, 4, 0, 0},
                                {8, 4, 0, 0}, {8, 8, 0, 0}, {8, 4, 4, 0}, {8, 8, 4, 0}, {8, 8, 8, 0},
                                {8, 8, 4, 4}, {8, 8, 8, 4}, {8, 8, 8, 8}};
    if (e < 0 || e > 12) return false;
    if (rmax >= 16) {
        for (int k = 0; k < 3; k++)
            if (t16[e][k]) out.push_back(t16[e][k]);
    } else {
        for (int k = 0; k < 4; k++)
            if (t8[e][k]) out.push_back(t8[e][k]);
    }
    return true;
}

// Plan for n = 2^a 3^b with first-stage radix r1 (a power of two >= 4 dividing n, with
// at least one more stage after it) and every other radix <= rmax.
bool build_plan(int n, int r1, int rmax, opo::AxisPlan &p, std::vector<cd> &tw)
{
    if (n < 8 || r1 < 4 || (r1 & (r1 - 1)) || n % r1 || n / r1 < 2) return false;
    int a = 0, b = 0, m = n / r1;
    while (m % 2 == 0) { m /= 2; a++; }
    while (m % 3 == 0) { m /= 3; b++; }
    if (m != 1) return false;
    std::vector<int> rad;
    rad.push_back(r1);
    for (int k = 0; k < b; k++) rad.push_back(3);
    if (!split_pow2(a, rmax, rad)) return false;
    if (rad.size() < 2 || (int)rad.size() > opo::kMaxStages) return false;
    p = opo::AxisPlan{};
    p.n = n;
    p.ns = (int)rad.size();
    tw.clear();
    int L = n;
    for (int s = 0; s < p.ns; s++) {
        const int R = rad[s], q = L / R;
        p.radix[s] = R;
        p.len[s] = L;
        p.twoff[s] = (int)tw.size();
        p.q[s] = make_fastdiv((unsigned)q);
        for (int k = 1; k < R; k++)
            for (int j = 0; j < q; j++) tw.push_back(std::polar(1.0, -2 * kPi * (double)j * k / L));
        L = q;
    }
    return L == 1;
}

// Frequency bin held at position pos after the forward (decimation-in-frequency)
// stages: pos = k1 (n/R1) + k2 (n/(R1 R2)) + ..., bin = k1 + R1 (k2 + R2 (k3 + ...)).
int bin_of_position(const opo::AxisPlan &p, int pos)
{
    int w = p.n, bin = 0, mult = 1;
    for (int s = 0; s < p.ns; s++) {
        w /= p.radix[s];
        const int k = pos / w;
        pos -= k * w;
        bin += k * mult;
        mult *= p.radix[s];
    }
    return bin;
}

// Centred index of FFT bin i on an n-point grid after the reference's fftshift
// (EFields3D.cuh:141-171): (i + n/2) mod n - n/2.
double centred(int i, int n) { return (double)((i + n / 2) % n) - 0.5 * n; }

enum PassKind { kT = 0, kX = 1, kY = 2 };

// Configuration of one pass kind: kernel variant, tile size, FFT plan, tile geometry
// and the device tables built for that plan ([0] crystal step, [1] round-trip
// boundary: GDD + mirrors for t, free space for x and y).
struct PassCfg {
    opo::PassVariant v{256, 16};
    size_t te = 0;
    opo::AxisPlan plan{};
    opo::TileGeom geo{};
    size_t smem = 0;  // one tile buffer (3 field regions)
    int grid = 0;     // CTAs of the single-instance kernel
    int line_nt = 0;  // t-pass: the line-specialised kernel's time axis (0: generic kernel)
    void *tw = nullptr;
    void *tab[2][3] = {};
    void *eom = nullptr;  // t-pass: EOM phase per time sample (natural order), or null
    // warp-specialised variant: ring arguments and the tensor maps of the fields
    // (t-pass: Api, Ap, As, Ai; y-pass: Ap, As, Ai)
    opo::WsArgs wsa{};
    CUtensorMap maps[4];
    std::vector<void *> allocs;
};

// Fused (x, y) plane pass: cluster size K (0: separate x and y passes), CTA size,
// first-stage radix of both axes, plans, geometry and tables ([0] crystal step, [1]
// free-space return).
struct PlaneCfg {
    int K = 0;
    int threads = 256;
    int r1 = 8;
    opo::AxisPlan px{}, py{};
    opo::TileGeom gx{}, gy{};
    opo::FastDiv rows{};
    unsigned regionA = 0;
    size_t smem = 0;
    void *twx = nullptr, *twy = nullptr;
    void *tabx[2][3] = {}, *taby[2][3] = {};
    std::vector<void *> allocs;
};

}  // namespace

struct OpoSolver {
    OpoParams p{};
    std::string err;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int dev = 0;
    size_t V = 0;
    size_t esz = 0;  // bytes per complex element
    void *field[4] = {};  // Api, Ap, As, Ai
    PassCfg pass[3];
    PlaneCfg plane;
    int *err_dev = nullptr;  // error word of the warp-specialised passes
    long long wait_cycles = 0;  // bound of their ring waits (0: the default ~2 s)
    // Set when a warp-specialised pass gave up a wait: that pass's tiles were not all
    // written, so the fields are lost.  Cleared once all four fields have been uploaded
    // again (reloaded: bit per field) or initialised (opo_init_fields).
    bool fields_lost = false;
    unsigned reloaded = 0;
    std::vector<double> w;
    double *partials = nullptr, *sums_dev = nullptr;
    int sum_blocks = 0;
    void *staging = nullptr;  // conversion buffer (V complex of the other precision)
    cudaGraphExec_t graph_rt[2] = {nullptr, nullptr};  // [last round trip?]
    int rt_index = 0;
    long long launches = 0;
    int launches_rt[2] = {0, 0};
    bool gdd_or_mirror = false;
    // streamed round trips (opo_stream_*): device stages of the four fields for the uploads
    // of the next run and the downloads of the last one, their copy streams and events
    struct Streamed {
        void *in[4] = {}, *out[4] = {};
        unsigned staged = 0;         // fields uploaded into `in` since the last run
        bool has_out = false;        // a run filled `out`
        cudaStream_t cs_in = nullptr, cs_out = nullptr;
        cudaEvent_t in_free = nullptr;   // compute stream: `in` copied into the fields
        cudaEvent_t in_ready = nullptr;  // cs_in: the uploads so far landed
        cudaEvent_t out_ready = nullptr; // compute stream: `out` holds the last run's fields
        cudaEvent_t out_free = nullptr;  // cs_out: the downloads so far left `out`
    } st;
    // per-pass event timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Timed { int kind; cudaEvent_t a, b; };
    std::vector<Timed> timed;
};

namespace {

const char *g_static_err = "";

int fail(OpoSolver *s, int code, const std::string &msg)
{
    if (s) s->err = msg;
    return code;
}

int cuda_fail(OpoSolver *s, cudaError_t e, const char *what)
{
    return fail(s, e == cudaErrorMemoryAllocation ? OPO_ERR_NOMEM : OPO_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define OPO_CU(s, call, what)                                   \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail((s), e_, what); \
    } while (0)

// After a synchronisation with the solver's stream: a warp-specialised pass that gave up
// on a bounded wait left a code in the error word (cleared here).
int check_pass_error(OpoSolver *s)
{
    if (!s->err_dev) return OPO_OK;
    int code = 0;
    OPO_CU(s, cudaMemcpy(&code, s->err_dev, sizeof(int), cudaMemcpyDeviceToHost), "error word");
    if (!code) return OPO_OK;
    cudaMemset(s->err_dev, 0, sizeof(int));
    s->fields_lost = true;
    s->reloaded = 0;
    return fail(s, OPO_ERR_CUDA, "a warp-specialised pass stopped after a pipeline wait timed out (code " +
                                     std::to_string(code) + "); the fields are lost until all four are uploaded "
                                     "again or initialised");
}

// Calls that read or advance the fields fail while they are lost (see fields_lost).
int require_fields(OpoSolver *s)
{
    if (!s->fields_lost) return OPO_OK;
    return fail(s, OPO_ERR_CUDA, "the fields were lost when a warp-specialised pass gave up a pipeline wait; "
                                 "upload all four (opo_set_field) or initialise them (opo_init_fields)");
}

cudaEvent_t take_event(OpoSolver *s)
{
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Brackets one kernel launch with events when pass timing is on.
struct PassTimer {
    OpoSolver *s;
    int kind;
    cudaEvent_t a = nullptr;
    PassTimer(OpoSolver *s_, int k) : s(s_), kind(k)
    {
        if (s->timing && (a = take_event(s))) cudaEventRecord(a, s->stream);
    }
    ~PassTimer()
    {
        if (!a) return;
        cudaEvent_t b = take_event(s);
        if (!b) { s->ev_pool.push_back(a); return; }
        cudaEventRecord(b, s->stream);
        s->timed.push_back({kind, a, b});
    }
};

template <typename C> C to_c(const cd &v);
template <> float2 to_c<float2>(const cd &v) { return make_float2((float)v.real(), (float)v.imag()); }
template <> double2 to_c<double2>(const cd &v) { return make_double2(v.real(), v.imag()); }

template <typename C> int upload(OpoSolver *s, std::vector<void *> &allocs, const std::vector<cd> &h, void **out)
{
    std::vector<C> tmp(h.size());
    for (size_t k = 0; k < h.size(); k++) tmp[k] = to_c<C>(h[k]);
    void *d = nullptr;
    OPO_CU(s, cudaMalloc(&d, sizeof(C) * (tmp.size() ? tmp.size() : 1)), "cudaMalloc(table)");
    allocs.push_back(d);
    if (!tmp.empty())
        OPO_CU(s, cudaMemcpy(d, tmp.data(), sizeof(C) * tmp.size(), cudaMemcpyHostToDevice), "cudaMemcpy(table)");
    *out = d;
    return OPO_OK;
}

int largest_divisor_leq(int n, int cap)
{
    if (cap < 1) return 0;
    for (int d = cap < n ? cap : n; d >= 1; d--)
        if (n % d == 0) return d;
    return 1;
}

void free_pass(PassCfg &pc)
{
    for (auto *a : pc.allocs) cudaFree(a);
    pc.allocs.clear();
    pc.tw = nullptr;
    pc.eom = nullptr;
    for (auto &row : pc.tab)
        for (auto &t : row) t = nullptr;
}

void free_plane(PlaneCfg &pc)
{
    for (auto *a : pc.allocs) cudaFree(a);
    pc = PlaneCfg{};
}

void drop_graphs(OpoSolver *s)
{
    for (auto &g : s->graph_rt)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            (void)cudaGetLastError();
    });
    return fn;
}

// Tensor map of one field viewed as a 3-D tensor (nx * m, ny, nt) of 8-byte elements,
// m = complex bytes / 8, with box (box0, box1, box2).
bool encode_field_map(CUtensorMap *map, void *field, int nx, int ny, int nt, size_t esz, unsigned box0,
                      unsigned box1, unsigned box2)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)nx * (esz / 8), (cuuint64_t)ny, (cuuint64_t)nt};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * esz, (cuuint64_t)nx * ny * esz};
    const cuuint32_t box[3] = {box0, box1, box2};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, field, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Diffraction factor tables of the x axis (xa) or the y axis in the digit-reversed order
// of plan pl: the propagator exp(sign L 2 pi^2 / k (fx^2 + fy^2)) of Solver3D.cuh:282-323
// factorised as (x factor)(y factor); fx = centred(i) / (dx nx).  crys[f] is the crystal
// step (the y factor carries exp(-alpha dz / 2)), free[f] the free-space return; the
// 1/(nx ny) normalisation is split as 1/nx, 1/ny (shipped 1/(nx ny nt) with OPO_ASIS_Q1).
void diffraction_tables(const OpoParams &p, bool xa, const opo::AxisPlan &pl, std::vector<cd> crys[3],
                        std::vector<cd> free[3])
{
    const int n = pl.n;
    const double q1scale = (!xa && (p.flags & OPO_ASIS_Q1)) ? 1.0 / p.nt : 1.0;
    for (int f = 0; f < 3; f++) {
        const double d = xa ? p.dx : p.dy;
        const double c = 2 * kPi * kPi / p.kdiff[f] / (d * n) / (d * n);
        crys[f].assign(n, cd(0, 0));
        free[f].assign(n, cd(0, 0));
        for (int pos = 0; pos < n; pos++) {
            const double u = centred(bin_of_position(pl, pos), n);
            cd v = std::polar(1.0, -p.dz * c * u * u) / (double)n;
            if (!xa) v *= std::exp(-0.5 * p.alpha[f] * p.dz) * q1scale;
            crys[f][pos] = v;
            free[f][pos] = std::polar(1.0, p.free_len * c * u * u) / (double)n;
        }
    }
}

// Default variant and tile size of a pass kind: 96 KB of shared memory for the three
// fields (4096 complex64 or 2048 complex128 per field), 256 threads.
void default_variant(bool fp64, int kind, opo::PassVariant &v, size_t &te)
{
    v.threads = 256;
    v.r1 = (fp64 && kind == kT) ? 8 : 16;
    te = fp64 ? 2048 : 4096;
}

// Build the plan, geometry and tables of one pass kind for variant v and tile size te.
template <typename C> int configure_pass(OpoSolver *s, int kind, opo::PassVariant v, size_t te)
{
    const OpoParams &p = s->p;
    const bool fp64 = sizeof(C) == 16;
    using TT = typename opo::TabOf<C>::type;
    if (!opo::variant_compiled(fp64, kind == kT, v)) return fail(s, OPO_ERR_INVALID, "kernel variant not compiled");
    if (kind != kT && !(p.flags & OPO_DIFFRACTION)) {
        // no (x, y) step: the pass never runs; keep the requested variant only
        drop_graphs(s);
        free_pass(s->pass[kind]);
        s->pass[kind] = PassCfg{};
        s->pass[kind].v = v;
        s->pass[kind].te = te;
        return OPO_OK;
    }
    PassCfg pc;
    pc.v = v;
    pc.te = te;
    const int nx = p.nx, ny = p.ny, nt = p.nt;
    const int n = kind == kT ? nt : (kind == kX ? nx : ny);
    if ((size_t)n > te) te = pc.te = (size_t)n;  // a tile holds at least one whole line
    std::vector<cd> tw;
    const int form = v.r1 & opo::kLineForm;
    int r1 = opo::radix_of(v);
    // line-specialised t-pass: a compiled time axis with its two-stage plan, whole tiles of
    // line_pixels() pixels, and every pixel transformed (not the shipped Q2 launch grid);
    // otherwise its generic fallback radix
    const int LP = opo::line_pixels(fp64);
    const bool line = form && kind == kT && opo::line_radix(nt) && nx % LP == 0 && !(p.flags & OPO_ASIS_Q2);
    if (line) r1 = opo::line_radix(nt);
    else if (form) r1 = opo::line_fallback_radix(fp64, v);
    else if (fp64 && kind == kT) r1 = std::min(r1, 8);  // 3 fields x r1 complex128 live in registers
    while (r1 >= 4 && !build_plan(n, r1, line ? 16 : opo::variant_max_radix(fp64, v), pc.plan, tw)) r1 /= 2;
    if (r1 < 4) return fail(s, OPO_ERR_INVALID, "grid sizes must be 2^a 3^b and >= 8");
    // a line variant keeps its setting (the bodies fix their radices); the fallback's
    // radix is checked by batches (solver_line_fallback_ok)
    pc.v.r1 = form ? v.r1 : r1;
    if (line && pc.plan.ns == 2) pc.line_nt = nt;
    const unsigned nxy = (unsigned)nx * ny;
    opo::TileGeom &g = pc.geo;
    if (pc.line_nt) {
        pc.te = (size_t)nt * LP;
        g.nlines = LP; g.ntiles = (nx / LP) * ny;
        g.lsl = 1; g.lsj = LP; g.region = (unsigned)(nt * LP);  // (the kernels lay out their own tiles)
        g.tdiv = make_fastdiv(nx / LP); g.tmulA = LP; g.tmulB = nx; g.gs_j = nxy; g.gs_l = 1;
        g.pairs = 1;
    } else if (kind == kT) {
        const int P = largest_divisor_leq(nx, (int)(te / nt));
        g.nlines = P; g.ntiles = (nx / P) * ny;
        g.lsl = 1; g.lsj = P; g.region = (unsigned)(nt * P);
        g.tdiv = make_fastdiv(nx / P); g.tmulA = P; g.tmulB = nx; g.gs_j = nxy; g.gs_l = 1;
        g.pairs = (P % 2 == 0 && nx % 2 == 0) ? 1 : 0;
    } else if (kind == kY) {
        const int Py = largest_divisor_leq(nx, (int)(te / ny));
        g.nlines = Py; g.ntiles = (nx / Py) * nt;
        g.lsl = 1; g.lsj = Py; g.region = (unsigned)(ny * Py);
        g.tdiv = make_fastdiv(nx / Py); g.tmulA = Py; g.tmulB = nxy; g.gs_j = nx; g.gs_l = 1;
        g.pairs = (Py % 2 == 0 && nx % 2 == 0) ? 1 : 0;
    } else {
        // x tiles: whole rows, stored row by row with an odd row stride nx + 1 so that
        // the line-parallel middle stages (consecutive threads on consecutive rows) and
        // the butterfly-parallel first and last stages are both bank-conflict free
        const int rows = largest_divisor_leq(ny * nt, (int)(te / nx));
        g.nlines = rows; g.ntiles = ny * nt / rows;
        g.lsl = (unsigned)(nx + 1); g.lsj = 1; g.region = (unsigned)(rows * (nx + 1));
        g.tdiv = make_fastdiv(1); g.tmulA = 0; g.tmulB = (unsigned)rows * nx; g.gs_j = 1; g.gs_l = nx;
    }
    const bool ws = opo::is_ws(v);
    if (kind != kX && !ws && !pc.line_nt && g.lsj * sizeof(C) < (fp64 ? 128u : 64u)) {
        // Line groups narrower than a shared-memory wavefront: the last forward stage's
        // butterflies (R rows apart, R its radix) would all fall on the same banks, so
        // one padding row follows every R rows.  Every earlier stage has a stride that
        // is a multiple of R, so its addressing stays affine.  FP32 line groups of 64 B
        // stay unpadded: that t-pass is issue-bound, and the index arithmetic and the
        // L1 space the padding takes cost more than the 2-way conflicts of that one
        // stage.  (The warp-specialised kernels keep the unpadded tile their tensor
        // copies write.)
        const int R = pc.plan.radix[pc.plan.ns - 1];
        if (R >= 2 && (R & (R - 1)) == 0) {
            unsigned sh = 0;
            while ((1 << sh) < R) sh++;
            g.psh = sh;
            g.region = (unsigned)(n + (n >> sh)) * g.lsj;
        }
    }
    g.nl = make_fastdiv((unsigned)g.nlines);
    g.rowlen = make_fastdiv((unsigned)nx);
    g.region = (g.region + 1u) & ~1u;  // keeps every field region 16-byte aligned
    if (ws) {
        // tensor / bulk copies land on 128-byte boundaries
        const unsigned per128 = (unsigned)(128 / sizeof(C));
        g.region = (g.region + per128 - 1) / per128 * per128;
    }
    pc.smem = pc.line_nt ? opo::tpass_line_smem(fp64, nt, r1) : 3 * (size_t)g.region * sizeof(C);
    if (pc.smem > 227 * 1024) return fail(s, OPO_ERR_INVALID, "tile does not fit in shared memory");
    if (ws) {
        opo::WsArgs &w = pc.wsa;
        const size_t es = sizeof(C);
        w = opo::WsArgs{};
        w.wait_cycles = s->wait_cycles;
        w.nstages = 2;
        w.stage_bytes = (unsigned)pc.smem;
        w.inner_mult = (unsigned)(es / 8);
        if (kind == kX) {
            if (((size_t)(nx + 1) * es) % 16 != 0)
                return fail(s, OPO_ERR_INVALID, "warp-specialised x-pass needs 16-byte row strides (FP64)");
            w.mode = opo::kWsRows;
            w.row_bytes = (unsigned)(nx * es);
            w.field_bytes = (unsigned)(g.nlines * nx * es);
        } else {
            const unsigned px = (unsigned)g.nlines, lines = (unsigned)n;
            if ((px * es) % 16 != 0 || ((size_t)nx * es) % 16 != 0)
                return fail(s, OPO_ERR_INVALID, "warp-specialised pass needs 16-byte tile rows");
            unsigned bl = lines < 256 ? lines : 256;
            while (lines % bl) bl--;
            if (bl < lines && ((size_t)bl * px * es) % 128 != 0)
                return fail(s, OPO_ERR_INVALID, "warp-specialised pass: box rows would start off 128-byte boundaries");
            w.mode = opo::kWsTensor;
            w.px = px;
            w.line_dim = kind == kT ? 2 : 1;
            w.lines = lines;
            w.box_lines = bl;
            w.field_bytes = (unsigned)(lines * px * es);
            const unsigned b0 = px * w.inner_mult;
            const int first = kind == kT ? 0 : 1;  // t-pass maps Api, Ap, As, Ai; y-pass Ap, As, Ai
            for (int k = first; k < 4; k++)
                if (!encode_field_map(&pc.maps[k - first], s->field[k], nx, ny, nt, es, b0, kind == kT ? 1 : bl,
                                      kind == kT ? bl : 1))
                    return fail(s, OPO_ERR_INVALID, "tensor map encoding failed");
        }
        pc.smem = opo::kWsHeaderBytes + w.nstages * (size_t)w.stage_bytes;
        if (pc.smem > 227 * 1024) return fail(s, OPO_ERR_INVALID, "stage ring does not fit in shared memory");
        if (kind != kT) {
            // the stage twiddles and up to three phase tables go into shared memory beside
            // the ring when that keeps as many CTAs resident per SM (228 KB per SM, 1 KB
            // reserved per CTA); otherwise the consumers read them from global memory
            const size_t tab_bytes = (tw.size() + 3 * (size_t)n) * sizeof(C);
            const size_t per_sm = 228 * 1024, with = pc.smem + tab_bytes;
            if (with <= 227 * 1024 && per_sm / (with + 1024) >= per_sm / (pc.smem + 1024)) {
                w.tab_off = (unsigned)pc.smem;
                w.ntw = (unsigned)tw.size();
                pc.smem = with;
            }
        }
    }

    int rc;
    if ((rc = upload<C>(s, pc.allocs, tw, &pc.tw))) { free_pass(pc); return rc; }
    const bool phys = (p.flags & OPO_PHYSICS) != 0;
    const opo::AxisPlan &pl = pc.plan;
    // FP32: every table of this plan carries the transform pair's gain compensation
    const std::vector<double> comp = fp64 ? std::vector<double>() : opo::fp32_pair_compensation(pl, tw);
    auto fix = [&](std::vector<cd> &t) {
        if (!comp.empty()) opo::scale_table(t, comp);
    };
    if (kind == kT) {
        // dispersion exp(i dz w (vinv + w b2/2)) exp(-alpha dz/2) / nt (Solver3D.cuh:153-169,
        // with the 1/nt of the inverse transform folded in); OPO_TOD adds w^3 b3/6 to the
        // phase (the crystals compute b3, PPLN.cuh:73, but the reference never applies it)
        const double q2scale = (p.flags & OPO_ASIS_Q2) ? 1.0 / ((double)nx * ny) : 1.0;
        for (int f = 0; f < 3; f++) {
            std::vector<cd> tab(nt);
            for (int pos = 0; pos < nt; pos++) {
                const double wk = s->w[bin_of_position(pl, pos)];
                const double b3 = (p.flags & OPO_TOD) ? p.beta3[f] : 0.0;
                cd v = std::polar(1.0, p.dz * wk * (p.vinv[f] + 0.5 * wk * p.beta2[f] + wk * wk * b3 / 6.0));
                if (!phys) v *= std::exp(-0.5 * p.alpha[f] * p.dz);
                tab[pos] = v * (q2scale / nt);
            }
            fix(tab);
            if ((rc = upload<TT>(s, pc.allocs, tab, &pc.tab[0][f]))) { free_pass(pc); return rc; }
        }
        // GDD compensation exp(i w^2 GDD / 2) (Solver3D.cuh:261-277, 676) times the mirror
        // sqrt(R) e^{i phase} (Cavity3D.cuh:12-28) for resonant signal / idler, / nt
        for (int f = 1; f < 3; f++) {
            const bool res = (p.resonant >> f) & 1u;
            const double R = f == 1 ? p.Rs : p.Ri;
            const cd mirror = res ? std::sqrt(R) * std::polar(1.0, p.detuning) : cd(1, 0);
            std::vector<cd> tab(nt);
            for (int pos = 0; pos < nt; pos++) {
                const double wk = s->w[bin_of_position(pl, pos)];
                tab[pos] = std::polar(1.0, 0.5 * wk * wk * p.gdd) * mirror / (double)nt;
            }
            fix(tab);
            if ((rc = upload<TT>(s, pc.allocs, tab, &pc.tab[1][f]))) { free_pass(pc); return rc; }
        }
        if (p.eom_beta != 0) {
            // EOM exp(i beta sin(2 pi fpm t)) on the t grid (Solver1D.cuh:63-72, t of
            // EFields3D.cuh:322-325), natural order
            std::vector<double> tt(nt);
            opo_time_freq(nt, p.t_window, tt.data(), nullptr);
            std::vector<cd> e(nt);
            for (int k = 0; k < nt; k++) e[k] = std::polar(1.0, p.eom_beta * std::sin(2 * kPi * p.eom_fpm * tt[k]));
            if ((rc = upload<C>(s, pc.allocs, e, &pc.eom))) { free_pass(pc); return rc; }
        }
    } else {
        std::vector<cd> crys[3], free[3];
        diffraction_tables(p, kind == kX, pl, crys, free);
        for (int f = 0; f < 3; f++) {
            fix(crys[f]);
            fix(free[f]);
        }
        for (int f = 0; f < 3; f++)
            if ((rc = upload<TT>(s, pc.allocs, crys[f], &pc.tab[0][f])) ||
                (rc = upload<TT>(s, pc.allocs, free[f], &pc.tab[1][f]))) {
                free_pass(pc);
                return rc;
            }
    }
    pc.grid = g.ntiles;
    if (ws) {
        // persistent: every resident CTA, at most one per tile
        int nsm = 0, per = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->dev);
        per = opo::ws_occupancy<C>(kind == kT, opo::PassVariant{v.threads - 32, pc.v.r1}, kind == kX, pc.smem);
        if (per < 1 || nsm < 1) {
            free_pass(pc);
            return fail(s, OPO_ERR_INVALID, "warp-specialised pass cannot be resident");
        }
        pc.grid = std::min(g.ntiles, per * nsm);
    }
    drop_graphs(s);
    free_pass(s->pass[kind]);
    s->pass[kind] = pc;
    return OPO_OK;
}

// Configure the fused (x, y) plane pass with clusters of K CTAs of `threads` threads and
// first-stage radix r1 on both axes (K = 0 selects the separate x and y passes).  A
// configuration that does not fit (grid not divisible by K, shared memory, no cluster
// of K resident) is refused with OPO_ERR_INVALID and leaves the current one in place.
template <typename C> int configure_plane(OpoSolver *s, int K, int threads, int r1)
{
    const OpoParams &p = s->p;
    const bool fp64 = sizeof(C) == 16;
    using TT = typename opo::TabOf<C>::type;
    if (K == 0) {
        drop_graphs(s);
        free_plane(s->plane);
        return OPO_OK;
    }
    if (K != 2 && K != 4 && K != 8) return fail(s, OPO_ERR_INVALID, "plane cluster size must be 0, 2, 4 or 8");
    if (!(p.flags & OPO_DIFFRACTION)) return fail(s, OPO_ERR_INVALID, "no diffraction step to fuse");
    if (!opo::plane_variant_compiled(threads)) return fail(s, OPO_ERR_INVALID, "plane kernel variant not compiled");
    const int nx = p.nx, ny = p.ny;
    if (nx % K || ny % K) return fail(s, OPO_ERR_INVALID, "nx and ny must be multiples of the plane cluster size");
    PlaneCfg pc;
    pc.K = K;
    pc.threads = threads;
    const int rmax = opo::plane_max_radix(fp64);
    std::vector<cd> twx, twy;
    int rx = r1, ry = r1;
    while (rx >= 4 && (rx > rmax || !build_plan(nx, rx, rmax, pc.px, twx))) rx /= 2;
    while (ry >= 4 && (ry > rmax || !build_plan(ny, ry, rmax, pc.py, twy))) ry /= 2;
    if (rx < 4 || ry < 4) return fail(s, OPO_ERR_INVALID, "grid sizes must be 2^a 3^b and >= 8");
    pc.r1 = std::max(rx, ry);
    const int rows = ny / K, ncol = nx / K;
    opo::TileGeom &gx = pc.gx;
    gx.nlines = rows; gx.ntiles = 0; gx.lsl = (unsigned)(nx + 1); gx.lsj = 1;
    gx.region = (unsigned)(rows * (nx + 1));
    gx.nl = make_fastdiv((unsigned)rows); gx.gs_j = 1; gx.gs_l = (unsigned)nx;
    opo::TileGeom &gy = pc.gy;
    gy.nlines = ncol; gy.ntiles = 0; gy.lsl = 1; gy.lsj = (unsigned)ncol; gy.region = (unsigned)(ny * ncol);
    gy.nl = make_fastdiv((unsigned)ncol); gy.gs_j = (unsigned)nx; gy.gs_l = 1;
    pc.rows = make_fastdiv((unsigned)rows);
    pc.regionA = (gx.region + 1u) & ~1u;  // column region 16-byte aligned
    pc.smem = ((size_t)pc.regionA + gy.region) * sizeof(C);
    if (pc.smem > 227 * 1024) return fail(s, OPO_ERR_INVALID, "plane slab does not fit in shared memory");
    if (opo::plane_max_clusters<C>(threads, K, pc.smem) < 1)
        return fail(s, OPO_ERR_INVALID, "no cluster of the plane pass can be resident");
    int rc;
    if ((rc = upload<C>(s, pc.allocs, twx, &pc.twx)) || (rc = upload<C>(s, pc.allocs, twy, &pc.twy))) {
        free_plane(pc);
        return rc;
    }
    std::vector<cd> crys[3], free[3];
    // FP32: the same gain compensation as the separate x / y passes' tables
    std::vector<double> comp;
    if (!fp64) comp = opo::fp32_pair_compensation(pc.px, twx);
    diffraction_tables(p, true, pc.px, crys, free);
    for (int f = 0; f < 3 && !comp.empty(); f++) {
        opo::scale_table(crys[f], comp);
        opo::scale_table(free[f], comp);
    }
    for (int f = 0; f < 3; f++)
        if ((rc = upload<TT>(s, pc.allocs, crys[f], &pc.tabx[0][f])) ||
            (rc = upload<TT>(s, pc.allocs, free[f], &pc.tabx[1][f]))) {
            free_plane(pc);
            return rc;
        }
    diffraction_tables(p, false, pc.py, crys, free);
    if (!fp64) comp = opo::fp32_pair_compensation(pc.py, twy);
    for (int f = 0; f < 3 && !comp.empty(); f++) {
        opo::scale_table(crys[f], comp);
        opo::scale_table(free[f], comp);
    }
    for (int f = 0; f < 3; f++)
        if ((rc = upload<TT>(s, pc.allocs, crys[f], &pc.taby[0][f])) ||
            (rc = upload<TT>(s, pc.allocs, free[f], &pc.taby[1][f]))) {
            free_plane(pc);
            return rc;
        }
    drop_graphs(s);
    free_plane(s->plane);
    s->plane = pc;
    return OPO_OK;
}

// Default plane pass: 256 threads, radix-8 first stages, the smallest cluster whose
// slab leaves room for two CTAs per SM (else the largest cluster that fits); the
// separate x and y passes when no cluster size fits the grid.
template <typename C> int default_plane(OpoSolver *s)
{
    if (!(s->p.flags & OPO_DIFFRACTION)) return configure_plane<C>(s, 0, 256, 8);
    int chosen = 0;
    for (int K : {2, 4, 8}) {
        const size_t esz = sizeof(C);
        if (s->p.nx % K || s->p.ny % K) continue;
        const size_t smem = ((size_t)(s->p.ny / K) * (s->p.nx + 1) + 1 + (size_t)s->p.ny * (s->p.nx / K)) * esz;
        if (smem > 227 * 1024) continue;
        chosen = K;
        if (smem <= 110 * 1024) break;
    }
    if (chosen && configure_plane<C>(s, chosen, 256, 8) == OPO_OK) return OPO_OK;
    s->err.clear();
    return configure_plane<C>(s, 0, 256, 8);
}

template <typename C> C *fld(OpoSolver *s, int k) { return static_cast<C *>(s->field[k]); }

template <typename C> typename opo::TabOf<C>::type *const *tabs(OpoSolver *s, int kind, int which)
{
    return reinterpret_cast<typename opo::TabOf<C>::type *const *>(s->pass[kind].tab[which]);
}

}  // namespace

namespace opo {

// Arguments of one t-pass of solver s: n_rk4 half steps (z of each given), then, for the
// fields in tmask, transform -> table `which_tab` (0 crystal, 1 round-trip boundary) ->
// inverse.
template <typename C>
TPassArgs<C> make_tpass_args(OpoSolver *s, bool reset_pump, int n_rk4, const double *zh, int which_tab,
                             unsigned tmask)
{
    const OpoParams &p = s->p;
    const PassCfg &pc = s->pass[kT];
    TPassArgs<C> a{};
    using T = typename TPassArgs<C>::T;
    for (int f = 0; f < 3; f++) a.f[f] = fld<C>(s, f + 1);
    a.psrc = reset_pump ? fld<C>(s, 0) : fld<C>(s, 1);
    a.g = pc.geo;
    a.plan = pc.plan;
    a.tw = static_cast<const C *>(pc.tw);
    for (int f = 0; f < 3; f++) a.tab[f] = tabs<C>(s, kT, which_tab)[f];
    a.tmask = tmask;
    a.n_rk4 = n_rk4;
    const bool phys = (p.flags & OPO_PHYSICS) != 0;
    const double h = 0.5 * p.dz;
    for (int f = 0; f < 3; f++) a.kappa[f] = (T)p.kappa[f];
    a.c1 = (T)(phys ? 0.5 * h : 0.5);
    a.c3 = (T)(phys ? h : 1.0);
    a.h6 = (T)(h / 6.0);
    for (int f = 0; f < 3; f++) {
        a.c1k[f] = (T)((phys ? 0.5 * h : 0.5) * p.kappa[f]);
        a.c3k[f] = (T)((phys ? h : 1.0) * p.kappa[f]);
        a.h6k[f] = (T)(h / 6.0 * p.kappa[f]);
    }
    a.use_phase = phys && p.dk != 0;
    for (int k = 0; k < n_rk4 && k < 2; k++) {
        // stage positions z, z + h/2, z + h (Solver3D.cuh:911-929 pass z, z+dz/4, z+dz/2)
        const double zs[3] = {zh[k], zh[k] + 0.5 * h, zh[k] + h};
        for (int j = 0; j < 3; j++) a.ph[k][j] = to_c<C>(std::polar(1.0, p.dk * zs[j]));
    }
    // the shipped quirk Q2 is the dispersion step's launch grid (Solver3D.cuh:603-629); the
    // closing pass's GDD compensation and mirrors act on every pixel (the mirror is a
    // transform over the whole field, Cavity3D.cuh:12-28)
    a.skip_rows = ((p.flags & OPO_ASIS_Q2) && which_tab == 0) ? 1 : 0;
    a.nx = (unsigned)p.nx;
    a.eom = which_tab == 1 ? static_cast<const C *>(pc.eom) : nullptr;
    a.line_nt = pc.line_nt;
    return a;
}

template <typename C> AxisArgs<C> make_axis_args(OpoSolver *s, int kind, int which_tab, unsigned mask)
{
    const PassCfg &pc = s->pass[kind];
    AxisArgs<C> a{};
    for (int f = 0; f < 3; f++) a.f[f] = fld<C>(s, f + 1);
    a.g = pc.geo;
    a.plan = pc.plan;
    a.tw = static_cast<const C *>(pc.tw);
    for (int f = 0; f < 3; f++) a.tab[f] = tabs<C>(s, kind, which_tab)[f];
    a.tmask = mask;
    return a;
}

}  // namespace opo

namespace {

template <typename C>
int enqueue_t(OpoSolver *s, bool reset_pump, int n_rk4, const double *zh, int which_tab, unsigned tmask)
{
    const PassCfg &pc = s->pass[kT];
    const opo::TPassArgs<C> a = opo::make_tpass_args<C>(s, reset_pump, n_rk4, zh, which_tab, tmask);
    PassTimer timer(s, 0);
    if (opo::is_ws(pc.v)) {
        opo::WsArgs w = pc.wsa;
        w.err = s->err_dev;
        const CUtensorMap maps[3] = {pc.maps[reset_pump ? 0 : 1], pc.maps[2], pc.maps[3]};
        OPO_CU(s, opo::launch_tpass_ws<C>(a, w, maps, opo::PassVariant{pc.v.threads - 32, pc.v.r1}, pc.grid, pc.smem,
                                          s->stream),
               "t-pass launch");
    } else if (opo::is_line(pc.v)) {
        OPO_CU(s, opo::launch_tpass_line<C>(a, pc.v, pc.line_nt, pc.plan.radix[0], pc.grid, pc.smem, s->stream),
               "t-pass launch");
    } else {
        OPO_CU(s, opo::launch_tpass<C>(a, opo::PassVariant{pc.v.threads, opo::radix_of(pc.v)}, pc.grid, pc.smem,
                                       s->stream),
               "t-pass launch");
    }
    s->launches++;
    return OPO_OK;
}

template <typename C> int enqueue_axis(OpoSolver *s, int kind, int which_tab, unsigned mask)
{
    const PassCfg &pc = s->pass[kind];
    const opo::AxisArgs<C> a = opo::make_axis_args<C>(s, kind, which_tab, mask);
    PassTimer timer(s, kind);
    if (opo::is_ws(pc.v)) {
        opo::WsArgs w = pc.wsa;
        w.err = s->err_dev;
        OPO_CU(s, opo::launch_axis_ws<C>(a, w, pc.maps, opo::PassVariant{pc.v.threads - 32, pc.v.r1}, kind == kX,
                                         pc.grid, pc.smem, s->stream),
               "axis-pass launch");
    } else {
        OPO_CU(s, opo::launch_axis<C>(a, pc.v, kind == kX, pc.grid, pc.smem, s->stream), "axis-pass launch");
    }
    s->launches++;
    return OPO_OK;
}

template <typename C> int enqueue_plane(OpoSolver *s, int which_tab, unsigned mask)
{
    using TT = typename opo::TabOf<C>::type;
    const PlaneCfg &pc = s->plane;
    const OpoParams &p = s->p;
    opo::PlaneArgs<C> a{};
    for (int k = 0; k < 3; k++) {
        a.f[k] = fld<C>(s, k + 1);
        a.tabx[k] = static_cast<const TT *>(pc.tabx[which_tab][k]);
        a.taby[k] = static_cast<const TT *>(pc.taby[which_tab][k]);
    }
    a.px = pc.px;
    a.py = pc.py;
    a.gx = pc.gx;
    a.gy = pc.gy;
    a.rows = pc.rows;
    a.twx = static_cast<const C *>(pc.twx);
    a.twy = static_cast<const C *>(pc.twy);
    a.tmask = mask;
    a.nx = (unsigned)p.nx;
    a.ny = (unsigned)p.ny;
    a.nt = (unsigned)p.nt;
    a.K = (unsigned)pc.K;
    a.regionA = pc.regionA;
    const unsigned planes = (unsigned)__builtin_popcount(mask) * (unsigned)p.nt;
    PassTimer timer(s, kX);
    OPO_CU(s, opo::launch_plane<C>(a, pc.threads, planes, pc.smem, s->stream), "plane-pass launch");
    s->launches++;
    return OPO_OK;
}

// The diffraction operator of a z-step (which_tab 0) or the free-space return (1) on
// the fields in mask: one fused plane pass, or the x then the y pass.
template <typename C> int enqueue_diffraction(OpoSolver *s, int which_tab, unsigned mask)
{
    if (s->plane.K) return enqueue_plane<C>(s, which_tab, mask);
    int rc;
    if ((rc = enqueue_axis<C>(s, kX, which_tab, mask))) return rc;
    return enqueue_axis<C>(s, kY, which_tab, mask);
}

// z of the first half step of step k (ref: the loop variable; physics: k dz).
double step_z(const OpoParams &p, int k) { return k * p.dz; }

// The crystal: for k in [0, n): RK4(h) D F RK4(h) (Solver3D.cuh:946-960), with
// D the t-axis operator and F the (x,y) one.  Passes: T(N D), X, Y, then for each
// later step T(N N D), X, Y; the final N is left to the caller.
template <typename C> int enqueue_crystal(OpoSolver *s, bool reset_pump)
{
    const OpoParams &p = s->p;
    const bool disp = (p.flags & OPO_DISPERSION) != 0, diff = (p.flags & OPO_DIFFRACTION) != 0;
    const bool phys = (p.flags & OPO_PHYSICS) != 0;
    int rc;
    for (int k = 0; k < p.n_steps; k++) {
        double zh[2];
        int nrk;
        if (k == 0) {
            zh[0] = step_z(p, 0);
            nrk = 1;
        } else {
            zh[0] = phys ? step_z(p, k - 1) + 0.5 * p.dz : step_z(p, k - 1);
            zh[1] = step_z(p, k);
            nrk = 2;
        }
        if ((rc = enqueue_t<C>(s, reset_pump && k == 0, nrk, zh, 0, disp ? 7u : 0u))) return rc;
        if (diff && (rc = enqueue_diffraction<C>(s, 0, 7u))) return rc;
    }
    return OPO_OK;
}

double last_half_z(const OpoParams &p)
{
    const int k = p.n_steps - 1;
    return (p.flags & OPO_PHYSICS) ? step_z(p, k) + 0.5 * p.dz : step_z(p, k);
}

template <typename C> int enqueue_single_pass(OpoSolver *s)
{
    int rc;
    if ((rc = enqueue_crystal<C>(s, false))) return rc;
    const double z = last_half_z(s->p);
    return enqueue_t<C>(s, false, 1, &z, 0, 0u);
}

// One round trip (Solver3D.cuh:979-997): fresh pump, crystal, final half step fused
// with GDD + mirrors on signal and idler (t-pass), then, unless this is the run's last
// round trip, the free-space return of signal and idler (x and y passes).  The free
// space and t-axis operators commute, so GDD + mirrors may precede the return.
template <typename C> int enqueue_round_trip(OpoSolver *s, bool last)
{
    const OpoParams &p = s->p;
    int rc;
    if ((rc = enqueue_crystal<C>(s, true))) return rc;
    const double z = last_half_z(p);
    if ((rc = enqueue_t<C>(s, false, 1, &z, 1, s->gdd_or_mirror ? 6u : 0u))) return rc;
    if (!last && (p.flags & OPO_DIFFRACTION) && (rc = enqueue_diffraction<C>(s, 1, 6u))) return rc;
    return OPO_OK;
}

template <typename C> int build_graph(OpoSolver *s, bool last)
{
    cudaGraph_t g = nullptr;
    OPO_CU(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    const long long before = s->launches;
    int rc = enqueue_round_trip<C>(s, last);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "end capture");
    s->launches_rt[last ? 1 : 0] = (int)(s->launches - before);
    s->launches = before;
    e = cudaGraphInstantiate(&s->graph_rt[last ? 1 : 0], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(s, e, "graph instantiate");
    return OPO_OK;
}

template <typename C> int run_round_trips(OpoSolver *s, int n)
{
    for (int k = 0; k < n; k++) {
        const bool last = s->rt_index == s->p.total_rt - 1;
        const int gi = last ? 1 : 0;
        if (s->timing) {
            int rc = enqueue_round_trip<C>(s, last);
            if (rc) return rc;
            s->rt_index++;
            continue;
        }
        if (!s->graph_rt[gi]) {
            int rc = build_graph<C>(s, last);
            if (rc) return rc;
        }
        OPO_CU(s, cudaGraphLaunch(s->graph_rt[gi], s->stream), "graph launch");
        s->launches += s->launches_rt[gi];
        s->rt_index++;
    }
    return OPO_OK;
}

template <typename C> int field_sums(OpoSolver *s, double out[3])
{
    {
        PassTimer timer(s, 3);
        OPO_CU(s, opo::launch_sums<C>(fld<C>(s, 1), fld<C>(s, 2), fld<C>(s, 3), s->V, s->partials,
                                      s->sum_blocks, s->sums_dev, s->stream),
               "sums launch");
    }
    s->launches += 2;
    OPO_CU(s, cudaMemcpyAsync(out, s->sums_dev, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "sums copy");
    OPO_CU(s, cudaStreamSynchronize(s->stream), "sums sync");
    if (int rc = check_pass_error(s)) return rc;
    for (int k = 0; k < 3; k++)
        if (!std::isfinite(out[k])) return fail(s, OPO_ERR_NONFINITE, "a field is not finite");
    return OPO_OK;
}

// ---------------------------------------------------------------------------------
// Autotuner: per pass kind, time every compiled variant x tile size that fits and keep
// the fastest.  Results are cached per (grid, precision, device) for the process.

struct TuneKey {
    int nx, ny, nt, prec, dev;
    bool operator==(const TuneKey &o) const
    {
        return nx == o.nx && ny == o.ny && nt == o.nt && prec == o.prec && dev == o.dev;
    }
};
struct TuneEntry {
    TuneKey key;
    opo::PassVariant v[3];
    size_t te[3];
    int plane[3];  // cluster size (0: separate x and y passes), threads, r1
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune_cache;

// Time per launch of `launch` (an enqueue returning an OPO code): 2 warm-up launches,
// then three rounds of 6, the best round's mean (one slow round -- a clock change, a
// neighbour's burst -- does not decide a candidate).
template <typename F> int time_launches(OpoSolver *s, F &&launch, float *ms)
{
    constexpr int warm = 2, reps = 6, rounds = 3;
    cudaEvent_t ev[rounds + 1] = {};
    int rc = OPO_OK;
    for (auto &e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = cuda_fail(s, cudaGetLastError(), "event");
    for (int r = 0; r < warm && !rc; r++) rc = launch();
    for (int k = 0; k < rounds && !rc; k++) {
        cudaEventRecord(ev[k], s->stream);
        for (int r = 0; r < reps && !rc; r++) rc = launch();
    }
    if (!rc) cudaEventRecord(ev[rounds], s->stream);
    cudaError_t e = rc ? cudaSuccess : cudaEventSynchronize(ev[rounds]);
    float best = 0;
    for (int k = 0; k < rounds && !rc && e == cudaSuccess; k++) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        if (k == 0 || t < best) best = t;
    }
    for (auto &x : ev)
        if (x) cudaEventDestroy(x);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(s, e, "autotune timing");
    *ms = best / reps;
    return OPO_OK;
}

template <typename C> int time_pass(OpoSolver *s, int kind, float *ms)
{
    const double zh[2] = {0, 0};
    return time_launches(s, [&] { return kind == kT ? enqueue_t<C>(s, false, 2, zh, 0, 7u) : enqueue_axis<C>(s, kind, 0, 7u); },
                         ms);
}

// Time of the diffraction operator (plane pass, or x then y pass), as time_launches.
template <typename C> int time_diffraction(OpoSolver *s, float *ms)
{
    return time_launches(s, [&] { return enqueue_diffraction<C>(s, 0, 7u); }, ms);
}

template <typename C> int autotune(OpoSolver *s)
{
    const bool fp64 = sizeof(C) == 16;
    const TuneKey key{s->p.nx, s->p.ny, s->p.nt, s->p.precision, s->dev};
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (auto &e : g_tune_cache)
            if (e.key == key) {
                for (int k = 0; k < 3; k++) {
                    int rc = configure_pass<C>(s, k, e.v[k], e.te[k]);
                    if (rc) return rc;
                }
                return configure_plane<C>(s, e.plane[0], e.plane[1], e.plane[2]);
            }
    }
    // The candidates are timed on scratch fields (zeroed, so no non-finite values), not on
    // the caller's: the fields are left as they were, as on a cache hit.  The guard puts
    // the caller's fields back and frees the scratch on every way out.
    struct ScratchFields {
        OpoSolver *s;
        void *mem = nullptr;
        void *saved[4] = {};
        ~ScratchFields()
        {
            if (!mem) return;
            for (int k = 0; k < 4; k++) s->field[k] = saved[k];
            cudaStreamSynchronize(s->stream);
            cudaFree(mem);
        }
    } scratch{s};
    OPO_CU(s, cudaMalloc(&scratch.mem, 4 * s->esz * s->V), "cudaMalloc(autotune scratch fields)");
    OPO_CU(s, cudaMemsetAsync(scratch.mem, 0, 4 * s->esz * s->V, s->stream), "memset(autotune scratch)");
    for (int k = 0; k < 4; k++) {
        scratch.saved[k] = s->field[k];
        s->field[k] = static_cast<char *>(scratch.mem) + k * s->esz * s->V;
    }
    TuneEntry best{key, {}, {}, {0, 256, 8}};
    const size_t tes[3] = {fp64 ? 512u : 1024u, fp64 ? 1024u : 2048u, fp64 ? 2048u : 4096u};
    const int threads[4] = {128, 256, 160, 288};  // 160 / 288: warp-specialised
    const int r1s[3] = {4, 8, 16};
    const long long launches0 = s->launches;
    for (int kind = 0; kind < 3; kind++) {
        float best_ms = 1e30f;
        best.v[kind] = s->pass[kind].v;
        best.te[kind] = s->pass[kind].te;
        if (kind != kT && !(s->p.flags & OPO_DIFFRACTION)) continue;
        for (size_t te : tes)
            for (int th : threads)
                for (int r1 : r1s) {
                    if (!opo::variant_compiled(fp64, kind == kT, opo::PassVariant{th, r1})) continue;
                    if (configure_pass<C>(s, kind, opo::PassVariant{th, r1}, te) != OPO_OK) continue;
                    if (s->pass[kind].v.r1 != r1) continue;  // plan fell back to a smaller radix
                    float ms = 0;
                    int rc = time_pass<C>(s, kind, &ms);
                    if (rc) return rc;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best.v[kind] = s->pass[kind].v;
                        best.te[kind] = te;
                    }
                }
        // line-specialised FP32 t-pass variants, where the grid has a compiled form
        for (int r1 : r1s) {
            const opo::PassVariant lv{128, r1 | opo::kLineForm};
            // one candidate per precision: its fallback radix (FP32 16, FP64 4) only matters
            // on grids without a line body
            if (kind != kT || !opo::variant_compiled(fp64, true, lv) || r1 != (fp64 ? 4 : 16)) continue;
            if (configure_pass<C>(s, kind, lv, tes[0]) != OPO_OK || !s->pass[kind].line_nt) continue;
            float ms = 0;
            int rc = time_pass<C>(s, kind, &ms);
            if (rc) return rc;
            if (ms < best_ms) {
                best_ms = ms;
                best.v[kind] = s->pass[kind].v;
                best.te[kind] = tes[0];
            }
        }
        int rc = configure_pass<C>(s, kind, best.v[kind], best.te[kind]);
        if (rc) return rc;
    }
    // diffraction: the tuned x and y passes against every plane-pass variant that fits
    if (s->p.flags & OPO_DIFFRACTION) {
        int rc = configure_plane<C>(s, 0, 256, 8);
        if (rc) return rc;
        float best_ms = 1e30f;
        if ((rc = time_diffraction<C>(s, &best_ms))) return rc;
        for (int K : {2, 4, 8})
            for (int th : {256, 512})
                for (int r1 : r1s) {
                    if (configure_plane<C>(s, K, th, r1) != OPO_OK) continue;
                    if (s->plane.r1 != r1) continue;  // plan fell back to a smaller radix
                    float ms = 0;
                    if ((rc = time_diffraction<C>(s, &ms))) return rc;
                    if (ms < best_ms) {
                        best_ms = ms;
                        best.plane[0] = K;
                        best.plane[1] = th;
                        best.plane[2] = r1;
                    }
                }
        s->err.clear();
        if ((rc = configure_plane<C>(s, best.plane[0], best.plane[1], best.plane[2]))) return rc;
    }
    s->launches = launches0;
    // back on the caller's fields: configure the chosen passes again, so that the tensor
    // maps of the warp-specialised kernels address those fields, not the scratch
    OPO_CU(s, cudaStreamSynchronize(s->stream), "autotune sync");
    for (int k = 0; k < 4; k++) s->field[k] = scratch.saved[k];
    for (int k = 0; k < 3; k++) {
        int rc = configure_pass<C>(s, k, best.v[k], best.te[k]);
        if (rc) return rc;
    }
    if (int rc = configure_plane<C>(s, best.plane[0], best.plane[1], best.plane[2])) return rc;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache.push_back(best);
    return OPO_OK;
}

bool valid_grid(int n) { return n >= 4; }
// x / y extent: >= 4, or 1 without diffraction (the plane-wave 1-D solver)
bool valid_extent(int n, unsigned flags) { return n >= 4 || (n == 1 && !(flags & OPO_DIFFRACTION)); }
// The pass kernels index a field with 32-bit arithmetic: at most 2^31 - 1 voxels.
bool valid_volume(int nx, int ny, int nt) { return (unsigned long long)nx * ny * nt <= 0x7fffffffull; }

}  // namespace

// =================================================================================
// C-ABI

extern "C" {

const char *opo_version(void) { return "cuopo3d-b200 0.1"; }

int opo_crystal_dispersion_pol(int crystal, double T, int extraordinary, double L, double out[4])
{
    Sellmeier m;
    if (!out || !sellmeier_of(crystal, T, extraordinary != 0, m) || !(L > 0)) return OPO_ERR_INVALID;
    out[0] = m.n(L);
    out[1] = m.vg(L);
    out[2] = m.gvd(L);
    // ZGP has no TOD in the reference: report the exact one
    out[3] = crystal == OPO_ZGP ? m.tod_exact(L) : m.tod(L);
    return OPO_OK;
}

int opo_crystal_dispersion(int crystal, double T, double L, double out[4])
{
    return opo_crystal_dispersion_pol(crystal, T, 1, L, out);
}

int opo_params_from_config(const OpoConfig *c, OpoParams *o, double *sc)
{
    if (!c || !o) return OPO_ERR_INVALID;
    if (!valid_extent(c->nx, c->flags) || !valid_extent(c->ny, c->flags) || !valid_grid(c->nt) || c->nz < 2 ||
        !valid_volume(c->nx, c->ny, c->nt))
        return OPO_ERR_INVALID;
    if (c->precision != OPO_FP32 && c->precision != OPO_FP64) return OPO_ERR_INVALID;
    CrystalModel m;
    if (!crystal_model(c->crystal, c->T, c->pol, m)) return OPO_ERR_INVALID;
    if (!(c->lp > 0) || !(c->ls > c->lp) || !(c->Lcr > 0) || !(c->LX > 0) || !(c->LY > 0)) return OPO_ERR_INVALID;
    const double lp = c->lp, ls = c->ls, li = ls * lp / (ls - lp);  // cuOPO3D.cu:17
    const double lam[3] = {lp, ls, li};
    double n[3], v[3], b2[3], b3[3], b3x[3], alpha[3];
    for (int f = 0; f < 3; f++) {
        n[f] = m.s[f].n(lam[f]);
        v[f] = m.s[f].vg(lam[f]);
        b2[f] = m.s[f].gvd(lam[f]);
        b3x[f] = m.s[f].tod_exact(lam[f]);
        b3[f] = c->crystal == OPO_ZGP ? b3x[f] : m.s[f].tod(lam[f]);
        alpha[f] = c->alpha[f] >= 0 ? c->alpha[f] : m.alpha[f];
    }
    const double dQ = c->dQ > 0 ? c->dQ : 2.0 * m.d33 / kPi;
    // a single pixel (1-D) has no transverse step: its pump sits at r = 0
    const double dx = c->nx > 1 ? c->LX / (c->nx - 1.0) : 0.0, dy = c->ny > 1 ? c->LY / (c->ny - 1.0) : 0.0,
                 dz = c->Lcr / (c->nz - 1.0);
    const bool phys = (c->flags & OPO_PHYSICS) != 0;
    // EFields3D.cuh:222-224 (and the crystal constructors): kp = 2 pi ns / lp and
    // ki = 2 pi ni / ls as shipped; corrected physics uses each wave's own n and lambda.
    const double kp = phys ? 2.0 * kPi * n[0] / lp : 2.0 * kPi * n[1] / lp;
    const double ks = 2.0 * kPi * n[1] / ls;
    const double ki = phys ? 2.0 * kPi * n[2] / li : 2.0 * kPi * n[2] / ls;
    // QPM crystals subtract the grating vector (PPLN.cuh:77); ZGP does not (ZGP.cuh:76)
    const double dk = kp - ks - ki - (m.qpm ? 2.0 * kPi / c->Lambda : 0.0);
    const double Lcav = c->Lcav > 0 ? c->Lcav : 4 * c->Lcr;
    const double trt = (Lcav + c->Lcr * (n[1] - 1)) / kC;  // Cavity3D.cuh:44
    const double dt = trt / (c->nt - 1);
    const int nsteps = c->n_steps > 0 ? c->n_steps : zloop_steps(c->Lcr, dz, c->zloop_f32 != 0);

    std::memset(o, 0, sizeof(*o));
    o->nx = c->nx; o->ny = c->ny; o->nt = c->nt; o->n_steps = nsteps;
    o->flags = c->flags; o->precision = c->precision;
    o->dz = (phys && c->n_steps > 0) ? c->Lcr / c->n_steps : dz;
    o->Lcr = c->Lcr; o->dx = dx; o->dy = dy;
    for (int f = 0; f < 3; f++) {
        o->kappa[f] = 2 * kPi * dQ / (n[f] * lam[f]);  // EFields3D.cuh:219-221
        o->beta2[f] = b2[f];
        o->beta3[f] = b3x[f];
        o->alpha[f] = alpha[f];
    }
    o->kdiff[0] = kp; o->kdiff[1] = ks; o->kdiff[2] = ki;
    o->vinv[0] = 1 / v[0] - 1 / v[2];  // Solver3D.cuh:163-165
    o->vinv[1] = 0.0;
    o->vinv[2] = 1 / v[2] - 1 / v[1];
    o->dk = dk;
    o->Rs = c->Rs; o->Ri = c->Ri; o->detuning = c->detuning;
    // Solver3D.cuh:676; GDD compensation exists only in the dispersion build (:476-480)
    o->gdd = (c->gdd_gamma != 0 && (c->flags & OPO_DISPERSION)) ? -c->gdd_gamma * b2[1] * c->Lcr : 0.0;
    o->free_len = c->Lcr;                                                // Solver3D.cuh:989
    o->resonant = c->resonant;
    o->total_rt = c->total_rt > 0 ? c->total_rt : 1;
    o->t_window = c->t_window > 0 ? c->t_window : trt;
    o->eom_beta = c->eom_beta;
    o->eom_fpm = c->eom_fpm;
    if (sc) {
        const double vals[OPO_N_SCALARS] = {n[0], n[1], n[2], v[0], v[1], v[2], b2[0], b2[1], b2[2],
                                            b3[0], b3[1], b3[2], dQ, dk, dx, dy, dz, kp, ks, ki,
                                            o->kappa[0], o->kappa[1], o->kappa[2], trt, dt, (double)nsteps};
        std::memcpy(sc, vals, sizeof(vals));
    }
    return OPO_OK;
}

int opo_power_cut_xy(const OpoConfig *cfg, const double sums[3], double power[3])
{
    if (!cfg || !sums || !power) return OPO_ERR_INVALID;
    OpoParams p;
    double sc[OPO_N_SCALARS];
    int rc = opo_params_from_config(cfg, &p, sc);
    if (rc) return rc;
    // Solver3D.cuh:534: 0.5 EPS0 C ns dx dy / (LX LY) sum |A|^2 (the signal index ns for
    // every field, as the reference)
    const double k = 0.5 * kEps0 * kC * sc[1] * p.dx * p.dy / (cfg->LX * cfg->LY);
    for (int f = 0; f < 3; f++) power[f] = k * sums[f];
    return OPO_OK;
}

int opo_time_freq(int nt, double T, double *t, double *w)
{
    if (nt < 2 || !(T > 0)) return OPO_ERR_INVALID;
    // Common.cuh:120-128 linspace, EFields3D.cuh:58-68 fftshift, :322-325
    for (int i = 0; t && i < nt; i++) t[i] = -T * 0.5 + i * (T * 0.5 - (-T * 0.5)) / (nt - 1);
    if (w) {
        const double fmin = -0.5 * nt / T, fmax = 0.5 * nt / T;
        const int c = nt / 2;
        for (int i = 0; i < nt; i++) {
            const int src = i < c ? i + c : i - c;
            w[i] = (fmin + src * (fmax - fmin) / (nt - 1)) * (2.0 * kPi);
        }
    }
    return OPO_OK;
}

int opo_pump_field(const OpoConfig *c, double *Api)
{
    OpoParams p;
    double sc[OPO_N_SCALARS];
    int rc = opo_params_from_config(c, &p, sc);
    if (rc) return rc;
    if (!Api) return OPO_ERR_INVALID;
    const int nx = c->nx, ny = c->ny, nt = c->nt;
    std::vector<double> t(nt);
    opo_time_freq(nt, p.t_window, t.data(), nullptr);
    const double np_ = sc[0], dx = p.dx, dy = p.dy, P = c->P, w0 = c->w0, w02 = w0 * w0;
    // EFields3D.cuh:247-253
    const double tau = c->FWHM * std::sqrt(2.0) / (2 * std::sqrt(2 * std::log(2.0)));
    const double zR = kPi * np_ * w02 / c->lp;
    const double eta = c->focal / zR;
    // 3-D peak 4P/(pi w0^2) (EFields3D.cuh:249); the plane-wave 1-D solver uses the mean
    // intensity 2P/(pi w0^2) (EFields1D.cuh:145-148) and has no focused modes
    const bool one_d = nx == 1 && ny == 1;
    if (one_d && (c->pump_mode == OPO_PUMP_FOCUSED_CW || c->pump_mode == OPO_PUMP_FOCUSED_PULSED ||
                  c->pump_mode == OPO_PUMP_FOCUSED_SECH2))
        return OPO_ERR_INVALID;
    const double pk = one_d ? 2.0 : 4.0;
    const double Ap0 = std::sqrt(pk * P / (kEps0 * kC * kPi * np_ * w02));
    const cd MX(1, -eta);
    // sech^2 intensity envelope (new): FWHM = 2 acosh(sqrt 2) ts; P is the window-average
    // power, so the peak power is P T / (2 ts).
    const double ts = c->FWHM / (2 * std::acosh(std::sqrt(2.0)));
    const double Ap0s = std::sqrt(pk * (P * p.t_window / (2 * ts)) / (kEps0 * kC * kPi * np_ * w02));
    const double uX = 0.5 * nx, uY = 0.5 * ny;
    for (int it = 0; it < nt; it++) {
        const double tn = t[it] / tau;
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const double rx = (x - uX) * dx, ry = (y - uY) * dy, r2 = rx * rx + ry * ry;
                const cd foc = (Ap0 / MX) * std::exp(cd(-r2, 0) / (w02 * MX));  // EFields3D.cuh:115
                cd v;
                switch (c->pump_mode) {
                case OPO_PUMP_WAVEPLANE_CW: v = Ap0 * std::exp(-r2 / w02); break;            // :79
                case OPO_PUMP_WAVEPLANE_PULSED: v = Ap0 * std::exp(-tn * tn - r2 / w02); break; // :96
                case OPO_PUMP_FOCUSED_CW: v = foc; break;
                case OPO_PUMP_FOCUSED_PULSED: v = foc * std::exp(-tn * tn); break;          // :132
                case OPO_PUMP_FOCUSED_SECH2: v = foc * (Ap0s / Ap0) / std::cosh(t[it] / ts); break;
                case OPO_PUMP_WAVEPLANE_SECH2: v = Ap0s * std::exp(-r2 / w02) / std::cosh(t[it] / ts); break;
                default: return OPO_ERR_INVALID;
                }
                const size_t id = (size_t)it * nx * ny + (size_t)y * nx + x;
                Api[2 * id] = v.real();
                Api[2 * id + 1] = v.imag();
            }
    }
    return OPO_OK;
}

int opo_noise(uint64_t seed, double sigma, size_t n, double *out)
{
    if (!out) return OPO_ERR_INVALID;
    for (size_t v = 0; v < 2 * n; v++) {
        double acc = 0;
        for (int j = 0; j < 12; j++) {
            uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(12 * v + j + 1);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            z ^= z >> 31;
            acc += (double)(z >> 11) * 0x1.0p-53;
        }
        out[v] = sigma * (acc - 6.0);
    }
    return OPO_OK;
}

static int create_impl(const OpoParams *p, const double *w, const opo::PassVariant *vv, const size_t *tt,
                       cudaStream_t ext_stream, OpoSolver **out)
{
    if (!out) return OPO_ERR_INVALID;
    *out = nullptr;
    if (!p || !w) return OPO_ERR_INVALID;
    if (p->precision != OPO_FP32 && p->precision != OPO_FP64) return OPO_ERR_INVALID;
    if (!valid_extent(p->nx, p->flags) || !valid_extent(p->ny, p->flags) || !valid_grid(p->nt) || p->n_steps < 1 ||
        !valid_volume(p->nx, p->ny, p->nt))
        return OPO_ERR_INVALID;
    OpoSolver *s = new (std::nothrow) OpoSolver();
    if (!s) return OPO_ERR_NOMEM;
    s->p = *p;
    if (s->p.total_rt < 1) s->p.total_rt = 1;
    s->w.assign(w, w + p->nt);
    s->V = (size_t)p->nx * p->ny * p->nt;
    s->esz = p->precision == OPO_FP64 ? sizeof(double2) : sizeof(float2);
    int rc = OPO_OK;
    cudaError_t e;
    do {
        if ((e = cudaGetDevice(&s->dev)) != cudaSuccess) { rc = cuda_fail(s, e, "cudaGetDevice"); break; }
        if (ext_stream) {
            s->stream = ext_stream;
            s->own_stream = false;
        } else if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess) {
            rc = cuda_fail(s, e, "stream");
            break;
        }
        for (int k = 0; k < 4 && !rc; k++) {
            if ((e = cudaMalloc(&s->field[k], s->esz * s->V)) != cudaSuccess) rc = cuda_fail(s, e, "cudaMalloc(field)");
            else if ((e = cudaMemset(s->field[k], 0, s->esz * s->V)) != cudaSuccess) rc = cuda_fail(s, e, "memset");
        }
        if (rc) break;
        // The attribute is per kernel function and shared by every solver of the process:
        // always allow the full 227 KB so no solver lowers it under another.
        if ((e = cudaMalloc((void **)&s->err_dev, sizeof(int))) != cudaSuccess ||
            (e = cudaMemset(s->err_dev, 0, sizeof(int))) != cudaSuccess) {
            rc = cuda_fail(s, e, "cudaMalloc(error word)");
            break;
        }
        if ((e = opo::configure_kernels(227 * 1024)) != cudaSuccess ||
            (e = opo::configure_plane_kernels(227 * 1024)) != cudaSuccess ||
            (e = opo::configure_ws_kernels(227 * 1024)) != cudaSuccess ||
            (e = opo::configure_line_kernels(227 * 1024)) != cudaSuccess) {
            rc = cuda_fail(s, e, "configure kernels");
            break;
        }
        for (int k = 0; k < 3 && !rc; k++) {
            opo::PassVariant v;
            size_t te;
            default_variant(p->precision == OPO_FP64, k, v, te);
            if (vv && tt) {
                v = vv[k];
                te = tt[k];
            }
            rc = p->precision == OPO_FP64 ? configure_pass<double2>(s, k, v, te) : configure_pass<float2>(s, k, v, te);
        }
        if (rc) break;
        if (!vv) {
            rc = p->precision == OPO_FP64 ? default_plane<double2>(s) : default_plane<float2>(s);
            if (rc) break;
        }
        s->gdd_or_mirror = s->p.gdd != 0 || (s->p.resonant & 6u);
        s->sum_blocks = 148 * 4;
        if ((e = cudaMalloc((void **)&s->partials, sizeof(double) * 3 * (s->sum_blocks + 1))) != cudaSuccess) {
            rc = cuda_fail(s, e, "cudaMalloc(partials)");
            break;
        }
        s->sums_dev = s->partials + 3 * s->sum_blocks;
    } while (0);
    if (rc) {
        g_static_err = "opo_create failed";
        std::fprintf(stderr, "opo_create: %s\n", s->err.c_str());
        opo_destroy(s);
        return rc;
    }
    *out = s;
    return OPO_OK;
}

int opo_create(const OpoParams *p, const double *w, OpoSolver **out)
{
    return create_impl(p, w, nullptr, nullptr, nullptr, out);
}

void opo_destroy(OpoSolver *s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &g : s->graph_rt)
        if (g) cudaGraphExecDestroy(g);
    for (auto &t : s->timed) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : s->ev_pool) cudaEventDestroy(e);
    for (cudaStream_t c : {s->st.cs_in, s->st.cs_out})
        if (c) {
            cudaStreamSynchronize(c);
            cudaStreamDestroy(c);
        }
    for (cudaEvent_t e : {s->st.in_free, s->st.in_ready, s->st.out_ready, s->st.out_free})
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < 4; k++) {
        if (s->st.in[k]) cudaFree(s->st.in[k]);
        if (s->st.out[k]) cudaFree(s->st.out[k]);
    }
    for (auto *f : s->field)
        if (f) cudaFree(f);
    if (s->partials) cudaFree(s->partials);
    if (s->staging) cudaFree(s->staging);
    if (s->err_dev) cudaFree(s->err_dev);
    for (auto &pc : s->pass) free_pass(pc);
    free_plane(s->plane);
    if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
}

static int ensure_staging(OpoSolver *s)
{
    if (s->staging) return OPO_OK;
    OPO_CU(s, cudaMalloc(&s->staging, sizeof(double2) * s->V), "cudaMalloc(staging)");
    return OPO_OK;
}

int opo_set_field(OpoSolver *s, int which, const void *src, int where, int prec)
{
    if (!s) return OPO_ERR_INVALID;
    if (which < 0 || which > 3 || !src || (where != OPO_MEM_HOST && where != OPO_MEM_DEVICE) ||
        (prec != OPO_FP32 && prec != OPO_FP64))
        return fail(s, OPO_ERR_INVALID, "opo_set_field: bad argument");
    const cudaMemcpyKind kind = where == OPO_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    s->reloaded |= 1u << which;
    if (s->reloaded == 0xfu) s->fields_lost = false;
    if (prec == s->p.precision) {
        OPO_CU(s, cudaMemcpyAsync(s->field[which], src, s->esz * s->V, kind, s->stream), "set_field copy");
        return OPO_OK;
    }
    int rc = ensure_staging(s);
    if (rc) return rc;
    const size_t sbytes = (prec == OPO_FP64 ? sizeof(double2) : sizeof(float2)) * s->V;
    OPO_CU(s, cudaMemcpyAsync(s->staging, src, sbytes, kind, s->stream), "set_field staging copy");
    if (prec == OPO_FP64)
        OPO_CU(s, opo::launch_convert_d2f((const double2 *)s->staging, (float2 *)s->field[which], s->V, s->stream), "convert");
    else
        OPO_CU(s, opo::launch_convert_f2d((const float2 *)s->staging, (double2 *)s->field[which], s->V, s->stream), "convert");
    s->launches++;
    return OPO_OK;
}

int opo_get_field(OpoSolver *s, int which, void *dst, int where, int prec)
{
    if (!s) return OPO_ERR_INVALID;
    if (which < 0 || which > 3 || !dst || (where != OPO_MEM_HOST && where != OPO_MEM_DEVICE) ||
        (prec != OPO_FP32 && prec != OPO_FP64))
        return fail(s, OPO_ERR_INVALID, "opo_get_field: bad argument");
    if (int rc = require_fields(s)) return rc;
    const cudaMemcpyKind kind = where == OPO_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (prec == s->p.precision) {
        OPO_CU(s, cudaMemcpyAsync(dst, s->field[which], s->esz * s->V, kind, s->stream), "get_field copy");
    } else {
        int rc = ensure_staging(s);
        if (rc) return rc;
        const size_t dbytes = (prec == OPO_FP64 ? sizeof(double2) : sizeof(float2)) * s->V;
        if (prec == OPO_FP64)
            OPO_CU(s, opo::launch_convert_f2d((const float2 *)s->field[which], (double2 *)s->staging, s->V, s->stream), "convert");
        else
            OPO_CU(s, opo::launch_convert_d2f((const double2 *)s->field[which], (float2 *)s->staging, s->V, s->stream), "convert");
        s->launches++;
        OPO_CU(s, cudaMemcpyAsync(dst, s->staging, dbytes, kind, s->stream), "get_field staging copy");
    }
    if (where == OPO_MEM_HOST) {
        OPO_CU(s, cudaStreamSynchronize(s->stream), "get_field sync");
        return check_pass_error(s);
    }
    return OPO_OK;
}

int opo_run_single_pass(OpoSolver *s)
{
    if (!s) return OPO_ERR_INVALID;
    if (int rc = require_fields(s)) return rc;
    return s->p.precision == OPO_FP64 ? enqueue_single_pass<double2>(s) : enqueue_single_pass<float2>(s);
}

int opo_run_round_trips(OpoSolver *s, int n)
{
    if (!s || n < 0) return s ? fail(s, OPO_ERR_INVALID, "negative round-trip count") : OPO_ERR_INVALID;
    if (int rc = require_fields(s)) return rc;
    return s->p.precision == OPO_FP64 ? run_round_trips<double2>(s, n) : run_round_trips<float2>(s, n);
}

int opo_run_round_trips_tallied(OpoSolver *s, int n, double *tallies, int *done)
{
    if (done) *done = 0;
    if (!s || n < 0) return s ? fail(s, OPO_ERR_INVALID, "negative round-trip count") : OPO_ERR_INVALID;
    if (int rc = require_fields(s)) return rc;
    for (int k = 0; k < n; k++) {
        int rc = s->p.precision == OPO_FP64 ? run_round_trips<double2>(s, 1) : run_round_trips<float2>(s, 1);
        if (rc) return rc;
        double sums[3];
        rc = s->p.precision == OPO_FP64 ? field_sums<double2>(s, sums) : field_sums<float2>(s, sums);
        if (done) *done = k + 1;
        if (tallies)
            for (int f = 0; f < 3; f++) tallies[3 * (size_t)k + f] = sums[f];
        if (rc == OPO_ERR_NONFINITE)
            return fail(s, OPO_ERR_NONFINITE, "Simulation failed: non-finite fields after round trip " +
                                                  std::to_string(s->rt_index));
        if (rc) return rc;
    }
    return OPO_OK;
}

// ---------------------------------------------------------------------------------
// Streamed round trips: uploads for the next run and downloads of the last run go through
// device stages on two copy streams, so they overlap the round trips on the compute
// stream.  Ordering (events): an upload waits until the previous run has taken `in`; a run
// waits for the uploads, copies `in` into the fields, runs, waits until the previous
// downloads left `out`, and copies the fields into `out`; a download waits for that run.

static int stream_setup(OpoSolver *s)
{
    auto &st = s->st;
    if (st.cs_in) return OPO_OK;
    OPO_CU(s, cudaStreamCreateWithFlags(&st.cs_in, cudaStreamNonBlocking), "stream create");
    OPO_CU(s, cudaStreamCreateWithFlags(&st.cs_out, cudaStreamNonBlocking), "stream create");
    for (cudaEvent_t *e : {&st.in_free, &st.in_ready, &st.out_ready, &st.out_free})
        OPO_CU(s, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event create");
    return OPO_OK;
}

int opo_stream_put(OpoSolver *s, int which, const void *host, int prec)
{
    if (!s) return OPO_ERR_INVALID;
    if (which < 0 || which > 3 || !host || prec != s->p.precision)
        return fail(s, OPO_ERR_INVALID, "opo_stream_put: bad argument (host data in the solver's precision)");
    if (int rc = stream_setup(s)) return rc;
    auto &st = s->st;
    const size_t bytes = s->esz * s->V;
    if (!st.in[which]) OPO_CU(s, cudaMalloc(&st.in[which], bytes), "cudaMalloc(stream stage)");
    OPO_CU(s, cudaStreamWaitEvent(st.cs_in, st.in_free, 0), "stream wait");
    OPO_CU(s, cudaMemcpyAsync(st.in[which], host, bytes, cudaMemcpyHostToDevice, st.cs_in), "stream upload");
    OPO_CU(s, cudaEventRecord(st.in_ready, st.cs_in), "event record");
    st.staged |= 1u << which;
    return OPO_OK;
}

int opo_stream_run(OpoSolver *s, int n)
{
    if (!s || n < 0) return s ? fail(s, OPO_ERR_INVALID, "negative round-trip count") : OPO_ERR_INVALID;
    if (int rc = stream_setup(s)) return rc;
    auto &st = s->st;
    const size_t bytes = s->esz * s->V;
    if (st.staged) {
        OPO_CU(s, cudaStreamWaitEvent(s->stream, st.in_ready, 0), "stream wait");
        for (int k = 0; k < 4; k++)
            if (st.staged & (1u << k)) {
                OPO_CU(s, cudaMemcpyAsync(s->field[k], st.in[k], bytes, cudaMemcpyDeviceToDevice, s->stream),
                       "stream stage copy");
                s->reloaded |= 1u << k;
            }
        OPO_CU(s, cudaEventRecord(st.in_free, s->stream), "event record");
        if (s->reloaded == 0xfu) s->fields_lost = false;
        st.staged = 0;
    }
    if (int rc = opo_run_round_trips(s, n)) return rc;
    OPO_CU(s, cudaStreamWaitEvent(s->stream, st.out_free, 0), "stream wait");
    for (int k = 0; k < 4; k++) {
        if (!st.out[k]) OPO_CU(s, cudaMalloc(&st.out[k], bytes), "cudaMalloc(stream stage)");
        OPO_CU(s, cudaMemcpyAsync(st.out[k], s->field[k], bytes, cudaMemcpyDeviceToDevice, s->stream),
               "stream stage copy");
    }
    OPO_CU(s, cudaEventRecord(st.out_ready, s->stream), "event record");
    st.has_out = true;
    return OPO_OK;
}

int opo_stream_get(OpoSolver *s, int which, void *host, int prec)
{
    if (!s) return OPO_ERR_INVALID;
    if (which < 0 || which > 3 || !host || prec != s->p.precision)
        return fail(s, OPO_ERR_INVALID, "opo_stream_get: bad argument (host data in the solver's precision)");
    auto &st = s->st;
    if (!st.has_out) return fail(s, OPO_ERR_INVALID, "opo_stream_get before any opo_stream_run");
    OPO_CU(s, cudaStreamWaitEvent(st.cs_out, st.out_ready, 0), "stream wait");
    OPO_CU(s, cudaMemcpyAsync(host, st.out[which], s->esz * s->V, cudaMemcpyDeviceToHost, st.cs_out),
           "stream download");
    OPO_CU(s, cudaEventRecord(st.out_free, st.cs_out), "event record");
    return OPO_OK;
}

int opo_stream_wait(OpoSolver *s)
{
    if (!s) return OPO_ERR_INVALID;
    auto &st = s->st;
    if (st.cs_in) OPO_CU(s, cudaStreamSynchronize(st.cs_in), "stream sync");
    OPO_CU(s, cudaStreamSynchronize(s->stream), "stream sync");
    if (st.cs_out) OPO_CU(s, cudaStreamSynchronize(st.cs_out), "stream sync");
    return check_pass_error(s);
}

int opo_set_wait_limit(OpoSolver *s, long long cycles)
{
    if (!s || cycles < 0) return s ? fail(s, OPO_ERR_INVALID, "negative wait limit") : OPO_ERR_INVALID;
    s->wait_cycles = cycles;
    for (auto &pc : s->pass) pc.wsa.wait_cycles = cycles;
    drop_graphs(s);  // captured launches hold the old bound
    return OPO_OK;
}

int opo_field_sums(OpoSolver *s, double sums[3])
{
    if (!s || !sums) return s ? fail(s, OPO_ERR_INVALID, "null output") : OPO_ERR_INVALID;
    if (int rc = require_fields(s)) return rc;
    return s->p.precision == OPO_FP64 ? field_sums<double2>(s, sums) : field_sums<float2>(s, sums);
}

int opo_synchronize(OpoSolver *s)
{
    if (!s) return OPO_ERR_INVALID;
    OPO_CU(s, cudaStreamSynchronize(s->stream), "synchronize");
    return check_pass_error(s);
}

int opo_set_pass_timing(OpoSolver *s, int enable)
{
    if (!s) return OPO_ERR_INVALID;
    s->timing = enable != 0;
    return OPO_OK;
}

int opo_pass_times(OpoSolver *s, double ms[4], long long counts[4])
{
    if (!s || !ms || !counts) return s ? fail(s, OPO_ERR_INVALID, "null output") : OPO_ERR_INVALID;
    OPO_CU(s, cudaStreamSynchronize(s->stream), "pass-times sync");
    for (int k = 0; k < 4; k++) { ms[k] = 0; counts[k] = 0; }
    for (auto &t : s->timed) {
        float v = 0;
        if (cudaEventElapsedTime(&v, t.a, t.b) == cudaSuccess) {
            ms[t.kind] += v;
            counts[t.kind]++;
        }
        s->ev_pool.push_back(t.a);
        s->ev_pool.push_back(t.b);
    }
    s->timed.clear();
    return OPO_OK;
}

int opo_init_fields(OpoSolver *s, const OpoConfig *cfg, uint64_t seed, double sigma, int idler_copy)
{
    if (!s || !cfg) return s ? fail(s, OPO_ERR_INVALID, "null configuration") : OPO_ERR_INVALID;
    int rc = opo::init_fields_device(s, cfg, seed, sigma, idler_copy, s->stream);
    if (!rc) {
        s->launches++;
        s->fields_lost = false;
        s->reloaded = 0xfu;
    }
    return rc;
}

int opo_autotune(OpoSolver *s)
{
    if (!s) return OPO_ERR_INVALID;
    return s->p.precision == OPO_FP64 ? autotune<double2>(s) : autotune<float2>(s);
}

int opo_set_tuning(OpoSolver *s, const int tuning[9])
{
    if (!s || !tuning) return OPO_ERR_INVALID;
    for (int k = 0; k < 3; k++) {
        const opo::PassVariant v{tuning[3 * k], tuning[3 * k + 2]};
        const size_t te = (size_t)tuning[3 * k + 1];
        int rc = s->p.precision == OPO_FP64 ? configure_pass<double2>(s, k, v, te) : configure_pass<float2>(s, k, v, te);
        if (rc) return rc;
    }
    return OPO_OK;
}

int opo_get_tuning(const OpoSolver *s, int out[9])
{
    if (!s || !out) return OPO_ERR_INVALID;
    for (int k = 0; k < 3; k++) {
        out[3 * k] = s->pass[k].v.threads;
        out[3 * k + 1] = (int)s->pass[k].te;
        out[3 * k + 2] = s->pass[k].v.r1;
    }
    return OPO_OK;
}

int opo_set_plane_pass(OpoSolver *s, int cluster, int threads, int r1)
{
    if (!s) return OPO_ERR_INVALID;
    return s->p.precision == OPO_FP64 ? configure_plane<double2>(s, cluster, threads, r1)
                                      : configure_plane<float2>(s, cluster, threads, r1);
}

int opo_get_plane_pass(const OpoSolver *s, int out[3])
{
    if (!s || !out) return OPO_ERR_INVALID;
    out[0] = s->plane.K;
    out[1] = s->plane.K ? s->plane.threads : 0;
    out[2] = s->plane.K ? s->plane.r1 : 0;
    return OPO_OK;
}

int opo_get_stream(const OpoSolver *s, void **stream)
{
    if (!s || !stream) return OPO_ERR_INVALID;
    *stream = (void *)s->stream;
    return OPO_OK;
}

int opo_round_trip_index(const OpoSolver *s) { return s ? s->rt_index : -1; }
long long opo_kernel_launches(const OpoSolver *s) { return s ? s->launches : -1; }
const char *opo_last_error(const OpoSolver *s) { return s ? s->err.c_str() : g_static_err; }

}  // extern "C"

namespace opo {

int solver_create_configured(const OpoParams *p, const double *w, const PassVariant v[3], const size_t te[3],
                             cudaStream_t stream, OpoSolver **out)
{
    return create_impl(p, w, v, te, stream, out);
}

PassVariant solver_pass_variant(const OpoSolver *s, int kind) { return s->pass[kind].v; }

bool solver_line_fallback_ok(const OpoSolver *s)
{
    const PassCfg &pc = s->pass[kT];
    if (!is_line(pc.v) || pc.line_nt) return true;
    return pc.plan.radix[0] == line_fallback_radix(s->p.precision == OPO_FP64, pc.v);
}

int solver_line_nt(const OpoSolver *s) { return s->pass[kT].line_nt; }

void solver_pass_info(const OpoSolver *s, int kind, int *ntiles, size_t *smem)
{
    *ntiles = s->pass[kind].geo.ntiles;
    *smem = s->pass[kind].smem;
}

const OpoParams &solver_params(const OpoSolver *s) { return s->p; }

size_t solver_device_bytes(const OpoSolver *s)
{
    size_t b = 4 * s->esz * s->V + 3 * sizeof(double) * (s->sum_blocks + 1);
    return b;
}

void *solver_field(OpoSolver *s, int which) { return s->field[which]; }

cudaStream_t solver_stream(const OpoSolver *s) { return s->stream; }

bool solver_gdd_or_mirror(const OpoSolver *s) { return s->gdd_or_mirror; }

void solver_tpass_z(const OpoParams &p, int tp, double zh[2], int *n_rk4)
{
    const bool phys = (p.flags & OPO_PHYSICS) != 0;
    if (tp == 0) {
        zh[0] = step_z(p, 0);
        zh[1] = 0;
        *n_rk4 = 1;
    } else if (tp < p.n_steps) {
        zh[0] = phys ? step_z(p, tp - 1) + 0.5 * p.dz : step_z(p, tp - 1);
        zh[1] = step_z(p, tp);
        *n_rk4 = 2;
    } else {
        zh[0] = last_half_z(p);
        zh[1] = 0;
        *n_rk4 = 1;
    }
}

int solver_fail(OpoSolver *s, int code, const char *msg) { return fail(s, code, msg); }

void solver_release_staging(OpoSolver *s)
{
    if (s->staging) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->staging);
        s->staging = nullptr;
    }
}

template TPassArgs<float2> make_tpass_args<float2>(OpoSolver *, bool, int, const double *, int, unsigned);
template TPassArgs<double2> make_tpass_args<double2>(OpoSolver *, bool, int, const double *, int, unsigned);
template AxisArgs<float2> make_axis_args<float2>(OpoSolver *, int, int, unsigned);
template AxisArgs<double2> make_axis_args<double2>(OpoSolver *, int, int, unsigned);

}  // namespace opo
