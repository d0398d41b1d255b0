// Complex helpers of the cuOPO3D headers used by programs (exp(i a), conjugate, |a|^2).
#pragma once

#include "DtypesConsts.cuh"

__host__ __device__ inline complex_t CpxExp(real_t a) { return make_cuFloatComplex(cosf(a), sinf(a)); }
__host__ __device__ inline complex_t CpxConj(complex_t a) { return make_cuFloatComplex(a.x, -a.y); }
__host__ __device__ inline real_t CpxAbs2(complex_t a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ inline real_t CpxAbs(complex_t a) { return sqrtf(CpxAbs2(a)); }
