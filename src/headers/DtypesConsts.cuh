// Types and grid constants of the drop-in headers.  As in cuOPO3D the grid is fixed at
// compile time; the defaults are cuOPO3D's 3-D ones (NX = NY = 128, NT = 2048 with
// -DDISPERSION, NZ = 100, NRT = 10000) and each can be overridden on the command line,
// e.g. -DOPO_NT=256 -DOPO_NRT=200.
#pragma once

#include "Libraries.cuh"

using real_t = float;
using complex_t = cuFloatComplex;  // the layout of cufftComplex
using rVech_t = thrust::host_vector<real_t>;
using rVecd_t = thrust::device_vector<real_t>;
using cVech_t = thrust::host_vector<complex_t>;
using cVecd_t = thrust::device_vector<complex_t>;

#ifndef OPO_NX
#define OPO_NX 128
#endif
#ifndef OPO_NY
#define OPO_NY OPO_NX
#endif
#ifndef OPO_NT
#ifdef DISPERSION
#define OPO_NT 2048
#else
#define OPO_NT 1
#endif
#endif
#ifndef OPO_NZ
#define OPO_NZ 100
#endif
#ifndef OPO_NRT
#define OPO_NRT 10000
#endif

const uint32_t NX = OPO_NX;
const uint32_t NY = OPO_NY;
const uint32_t NT = OPO_NT;
const uint32_t SIZE = NX * NY * NT;
const uint32_t NZ = OPO_NZ;
const uint32_t NRT = OPO_NRT;
const uint32_t BLKT = 1 << 5;
const uint32_t BLKX = 1 << 4;
const uint32_t BLKY = BLKX;

const real_t PI = 3.14159265358979323846;
const real_t C = 299792458 * 1E6 / 1E12;           // speed of light [um/ps]
const real_t EPS0 = 8.8541878128E-12 * 1E12 / 1E6; // vacuum permittivity [W ps / (V^2 um)]
