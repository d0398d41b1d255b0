// Drop-in header set for programs written against the cuOPO3D headers: the classes keep
// their names, constructor arguments and public members, and the split-step runs in the
// cuopo3d-b200 library (include/cuopo3d.h) instead of header-only cuFFT kernels.
// This file pulls in the standard, CUDA runtime and Thrust headers those programs use.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <tuple>
#include <unordered_set>
#include <vector>

#include <cuComplex.h>
#include <cuda_runtime.h>
#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
