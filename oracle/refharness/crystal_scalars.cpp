// Test infrastructure: prints the dispersion scalars (n, group velocity, GVD, TOD)
// computed by the reference's own crystal classes (src/headers/CrystalsBase/*.cuh, host
// code only, read where they lie) as JSON lines, so the oracle and the library can be
// pinned against them.  Built by build_crystal_scalars.sh with the headers' float math
// mapped to double (real_t = double, sqrtf -> sqrt, powf -> pow), like the FP64 solver
// harness.  Usage: crystal_scalars > scalars.jsonl
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>
#include <tuple>

typedef double real_t;
typedef unsigned int uint;
#define sqrtf sqrt
#define powf pow
// reference constants, src/headers/DtypesConsts.cuh:55-57
const real_t PI = 3.14159265358979323846;
const real_t C = 299792458 * 1E6 / 1E12;
#define NX 16
#define NY 16
#define NZ 16
static void printLineOnScreen() {}
using std::tie;

#include "CrystalsBase/PPLN.cuh"
#include "CrystalsBase/MgOPPLN.cuh"
#include "CrystalsBase/MgOsPPLT.cuh"
#include "CrystalsBase/ZGP.cuh"

template <class Cr> void qpm(const char *name, int id, double T, double L)
{
    Cr c(800.0, 800.0, 5000.0, T, 7.0, L, 2 * L, 2 * L);
    std::printf("{\"crystal\": \"%s\", \"id\": %d, \"T\": %.17g, \"pol\": \"\", \"lambda\": %.17g, "
                "\"n\": %.17g, \"vg\": %.17g, \"b2\": %.17g, \"b3\": %.17g}\n",
                name, id, T, L, c.n(L, T), c.GV(L, T), c.GVD(L, T), c.TOD(L, T));
}

void zgp(double L, char pol)
{
    ZGP c(800.0, 800.0, 5000.0, std::make_tuple(pol, pol, pol), L, 2 * L, 2 * L);
    std::printf("{\"crystal\": \"ZGP\", \"id\": 3, \"T\": 0, \"pol\": \"%c\", \"lambda\": %.17g, "
                "\"n\": %.17g, \"vg\": %.17g, \"b2\": %.17g, \"b3\": null}\n",
                pol, L, c.n(L, pol), c.GV(L, pol), c.GVD(L, pol));
}

int main()
{
    std::cout.setstate(std::ios_base::failbit);  // the constructors print their banners
    const double Ts[] = {20.0, 27.0, 60.0, 100.0};
    const double Ls[] = {0.532, 0.8, 1.064, 1.55, 2.1, 3.2};
    for (double T : Ts)
        for (double L : Ls) {
            qpm<PPLN>("PPLN", 0, T, L);
            qpm<MgOsPPLT>("MgOsPPLT", 1, T, L);
            qpm<MgOPPLN>("MgOPPLN", 2, T, L);
        }
    const double Lz[] = {2.0, 2.5, 3.2, 4.0, 6.4, 8.0};
    for (double L : Lz) {
        zgp(L, 'o');
        zgp(L, 'e');
    }
    return 0;
}
