// The drop-in header set: programs written against cuOPO3D's headers include
// "headers/Libraries.cuh" and "headers/PackageLibraries.cuh" and link -lcuopo3d.
#pragma once

#include "DtypesConsts.cuh"
#include "Common.cuh"
#include "Files.cuh"
#include "Operators.cuh"
#include "Crystals.cuh"
#include "EFields3D.cuh"
#include "Cavity3D.cuh"
#include "Solver3D.cuh"
